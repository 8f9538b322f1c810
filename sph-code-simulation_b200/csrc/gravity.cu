// gravity.cu — GravityForce::calculation (Barnes–Hut tree walk and the
// exhaustive direct sum).
//
// Reference: src/gravity_force.cpp:52-89, BHNode::calc_force
// (src/bhtree.cpp:347-393) and the Hernquist & Katz softening kernels f, g
// (src/bhtree.cpp:318-345).
//
// Per-lane stackless walk over the preorder node array: each lane (one
// particle; a warp holds 32 octree-consecutive particles) either accepts its
// current node as an (unsoftened) monopole and jumps over the subtree (skip
// pointer), or opens it — a leaf is then summed pairwise with spline-softened
// f and g and skipped, an internal node is descended into (index + 1).  Lanes
// follow their own paths, so a warp runs as many iterations as its longest
// walk rather than the union of its lanes' walks (1.5x faster on the Evrard
// sphere than a warp-synchronous union walk).  Each lane meets its nodes in
// exactly the order of the reference's recursion and adds into acc (starting
// from the fluid acceleration) in that order, so in the plain form with
// unfused FP64 (-fmad=false for this file) the result is bit-identical to the
// reference's on the same tree.  The mixed-precision walk is in
// gravity_mixed.cu (compiled with FMA contraction).
// The softened leaf pairs are 1.4 % of a particle's interactions on the 8.78 M
// Evrard sphere but a third of the walk's time (116 ms per step with them,
// 77 ms with their arithmetic left out, a timing-only copy): each one runs
// the reference's IEEE divisions on one lane while the warp waits.  Measured
// and not kept: walking each warp's path in segments, recording the opened
// leaves' pairs, computing their terms with all 32 lanes and replaying the
// segment to add every term in the reference's order (bit-identical, 190 ms:
// the second pass over the nodes costs more than the divergence it removes);
// lanes that park on an opened leaf until 5 / 10 / 16 lanes are parked and
// then compute their next pairs together (169 / 225 / 286 ms: parked lanes
// idle far longer than the divergent pairs take); the square roots and
// divisions formed from the hardware rsqrt / rcp estimates (about 2^-20) with
// a Newton step each, every rounding proven by a fused multiply-add residual
// test (Tuckerman's) and the IEEE operations taken only when the test could
// not prove it (bit-identical on all 8.78 M particles; 126.0 ms with the
// monopoles alone, 156.8 ms with the leaf pairs too, against 112.0 ms: the
// proof costs more issue slots than the IEEE sequences it replaces); an
// accepted node's monopole terms formed one iteration later, beside the next
// node's opening test (bit-identical; 134.1 ms under a branch, 141.7 ms
// unconditional with selects: 103 registers against 92, fewer warps in
// flight).  Kept: the squared edge of
// each level from a table in shared memory instead of an ldexp per node, and
// the next node's records loaded as soon as the opening test has chosen it
// (116.0 -> 114.9 ms together; capped at 6 resident blocks the prefetching
// walk spills and takes 124.8 ms).  The walk waits on its FP64 dependency
// chains (the correctly rounded square roots and divisions), not on loads.
#include <cuda_runtime.h>

#include "context.cuh"
#include "softening.cuh"

namespace sphgpu {

namespace {

// one warp per block: 113.5 -> 112.0 ms against 128 (256: 130.5 ms).  The walk
// takes 92 registers (21 resident warps per SM); capped for 24 / 28 warps it
// spills and takes 129.0 / 172.5 ms.
constexpr int GBLK = 32;

// subset != null: only the listed particles (the mixed form's FP64
// re-evaluation); those launches add to no work counter.
__global__ void __launch_bounds__(GBLK) k_gravity(DevParams P, DevState S, DevTree Tr, int n,
                                                  DevStatus* __restrict__ st, const int* __restrict__ subset,
                                                  int nsub)
{
    const int slot = blockIdx.x * GBLK + threadIdx.x;
    const bool valid = slot < (subset ? nsub : n);
    const int i = subset ? (valid ? subset[slot] : n) : slot;
    double xi = 0, yi = 0, zi = 0, hi = 1;
    double4 acc = make_double4(0, 0, 0, 0);
    if(valid) {
        const double4 p = S.pos[i];
        xi = p.x;
        yi = p.y;
        zi = p.z;
        hi = S.vel[i].w;
        acc = S.acc[i];
    }
    double ax = acc.x, ay = acc.y, az = acc.z, phi = 0.0;
    const double G = P.G;
    const int nnodes = *Tr.nnodes;
    // node edges halve exactly per level: edge(L) = root edge * 2^(1 - L);
    // the squared edge of every level, as the opening test forms it
    __shared__ double s_l2[256];
    {
        const double root_edge = ldg4(&Tr.geo[0]).w;
        for(int L = threadIdx.x; L < 256; L += GBLK) {
            const double e = ldexp(root_edge, 1 - L);
            s_l2[L] = e * e;
        }
        __syncthreads();
    }
    int nd = valid ? 0 : nnodes, steps = 0;
    unsigned n_mono = 0, n_leaf = 0;  // work counters of this lane (steps = nodes met)
    // the records of the node in hand; the next node's are loaded as soon as
    // the opening test has chosen it, before this node's terms are formed
    int4 lk = make_int4(0, 0, nnodes, 0);
    double4 mc = make_double4(0, 0, 0, 0);
    if(nd < nnodes) {
        lk = __ldg(&Tr.link[nd]);
        mc = ldg4(&Tr.mass[nd]);
    }
    while(nd < nnodes) {
        if(++steps > nnodes) {  // corrupt node table: report, never loop
            atomicOr(&st->pass_guard, PASS_GUARD_GRAVITY);
            break;
        }
        const bool leaf = (lk.w >> 8) != 0;
        const Vec3d d = rij(P, xi, yi, zi, mc.x, mc.y, mc.z);
        const double l2 = s_l2[lk.w & 0xff];
        const double d2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const bool open = (l2 > P.theta2 * d2) || (d2 < l2);
        const int next = (open && !leaf) ? nd + 1 : lk.z;
        int4 lk_n = lk;
        double4 mc_n = mc;
        if(next < nnodes) {
            lk_n = __ldg(&Tr.link[next]);
            mc_n = ldg4(&Tr.mass[next]);
        }
        if(!open) {
            ++n_mono;
            const double rinv = 1.0 / sqrt(d2);
            phi -= G * mc.w * rinv;
            const double s = G * mc.w * (rinv * rinv * rinv);
            ax -= d.x * s;
            ay -= d.y * s;
            az -= d.z * s;
        }
        if(open && leaf) {
            n_leaf += (unsigned)(lk.y - lk.x) - ((i >= lk.x && i < lk.y) ? 1u : 0u);
            for(int q = lk.x; q < lk.y; ++q) {
                if(q == i) continue;
                const double4 pq = ldg4(&S.pos[q]);
                const double hq = __ldg(&S.vel[q].w);
                const Vec3d r = rij(P, xi, yi, zi, pq.x, pq.y, pq.z);
                const double rr = sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
                phi -= G * pq.w * (hk_f<double>(rr, hi) + hk_f<double>(rr, hq)) * 0.5;
                const double c = G * pq.w * (hk_g<double>(rr, hi) + hk_g<double>(rr, hq)) * 0.5;
                ax -= r.x * c;
                ay -= r.y * c;
                az -= r.z * c;
            }
        }
        nd = next;
        lk = lk_n;
        mc = mc_n;
    }
    if(valid) {
        S.acc[i] = make_double4(ax, ay, az, acc.w);
        S.visc[i].w = phi;
    }
    if(subset) return;
    block_count(&st->grav_nodes, (unsigned)min(steps, nnodes));
    block_count(&st->grav_mono, n_mono);
    block_count(&st->grav_leaf_pairs, n_leaf);
}

// -DEXHAUSTIVE_SEARCH direct summation (src/gravity_force.cpp:70-84): every j
// in caller-index order, self included.
__global__ void k_gravity_direct(DevParams P, DevState S, int n, const int* __restrict__ inv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const double4 p = S.pos[i];
    const double hi = S.vel[i].w;
    const double G = P.G;
    double phi = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
    for(int jid = 0; jid < n; ++jid) {
        const int j = inv[jid];
        const double4 pj = S.pos[j];
        const double hj = S.vel[j].w;
        const Vec3d r = rij(P, p.x, p.y, p.z, pj.x, pj.y, pj.z);
        const double rr = sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
        phi -= G * pj.w * (hk_f<double>(rr, hi) + hk_f<double>(rr, hj)) * 0.5;
        const double c = G * pj.w * (hk_g<double>(rr, hi) + hk_g<double>(rr, hj)) * 0.5;
        fx -= r.x * c;
        fy -= r.y * c;
        fz -= r.z * c;
    }
    double4 a = S.acc[i];
    a.x += fx;
    a.y += fy;
    a.z += fz;
    S.acc[i] = a;
    S.visc[i].w = phi;
}

}  // namespace

int gravity(sphgpu_ctx* c, bool direct)
{
    // the mixed form's FP64 re-evaluation follows the last module that
    // writes acc (recheck.cu); GravityForce runs every step, with gravity off too
    if(!c->prm.use_gravity) return direct ? SPHGPU_OK : mixed_recheck(c);
    if(!direct && !c->have_tree) return fail(c, SPHGPU_ERR_STATE, "GravityForce before tree make");
    if(!direct && c->prm.precision == SPHGPU_MIXED) {
        // the walk's FP32 node records: tree data, timed with the tree
        stage_begin(c, SPHGPU_T_TREE);
        const int rc = gravity_nodes_mixed(c);
        if(rc < 0) return rc;
        stage_end(c, SPHGPU_T_TREE, 1);
    }
    stage_begin(c, SPHGPU_T_GRAVITY);
    if(direct) {
        k_gravity_direct<<<grid_for(c->n, 128), 128, 0, c->stream>>>(c->dp, c->s, c->n, c->d_inv);
    } else if(c->prm.precision == SPHGPU_MIXED) {
        const int rc = gravity_walk_mixed(c);
        if(rc < 0) return rc;
    } else {
        k_gravity<<<grid_for(c->n, GBLK), GBLK, 0, c->stream>>>(c->dp, c->s, c->t, c->n, c->d_status, nullptr, 0);
    }
    SPHGPU_LAUNCH_CHECK(c, "GravityForce");
    stage_end(c, SPHGPU_T_GRAVITY, 1);
    return direct ? SPHGPU_OK : mixed_recheck(c);
}

int gravity_subset64(sphgpu_ctx* c, const int* idx, int nsub)
{
    if(!c->prm.use_gravity || nsub <= 0) return SPHGPU_OK;
    k_gravity<<<grid_for(nsub, GBLK), GBLK, 0, c->stream>>>(c->dp, c->s, c->t, c->n, c->d_status, idx, nsub);
    SPHGPU_LAUNCH_CHECK(c, "GravityForce (FP64 re-evaluation)");
    return SPHGPU_OK;
}

}  // namespace sphgpu
