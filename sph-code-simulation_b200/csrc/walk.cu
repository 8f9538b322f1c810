// walk.cu — batched BHTree::neighbor_search and exhaustive_search.
//
// Reference: BHNode::neighbor_search (src/bhtree.cpp:277-316) — per node, the
// L-infinity box test |d_k| <= edge/2 + h against the node centre, then at a
// leaf the radius test r^2 < h^2 on every particle of the leaf list, with
// h = sml (gather) or max(sml, node.kernel_size) (is_ij).
//
// Warp-cooperative walk: a warp owns 32 consecutive particles in octree order
// (spatially coherent) and scans the preorder node array once.  Each lane
// keeps one bit per tree level: bit L says "my box test passed at the current
// level-L ancestor".  A node at level L is live for a lane iff bits 1..L-1 are
// all set — exactly the set of nodes the reference's recursion would visit
// for that particle.  The warp descends into a node (index + 1) when any live
// lane passes, else jumps over the subtree (skip pointer).  Every test is
// evaluated in unfused FP64 (this file builds with -fmad=false) so each
// lane's list equals the reference's list as a set, and even in order before
// the reference's distance sort.
//
// Lists go to an ELL buffer (capacity slots per particle, row-major).  A list
// longer than the capacity is counted but not stored; the host grows the
// buffer and re-runs (status.overflow).  More than neighbor_number * 1000
// entries is the reference's fatal overflow (src/bhtree.cpp:129-135).
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int WBLK = 128;

// Per-lane walk of one particle (lane) over the preorder node array; the
// caller's warp runs it in lock step.  Returns the list length.
template <bool IJ>
__device__ __forceinline__ int walk_lanes(const DevParams& P, const DevState& S, const DevTree& T, bool valid,
                                          double xi, double yi, double zi, double hi, int* __restrict__ list,
                                          size_t row, int cap, DevStatus* __restrict__ st)
{
    const int nnodes = *T.nnodes;
    int cnt = 0;
    unsigned bits = 0;
    int nd = 0, steps = 0;
    while(nd < nnodes) {
        // a preorder scan visits each node at most once; more means a corrupt
        // node table: stop and report instead of looping
        if(++steps > nnodes) {
            st->guard = 1;
            break;
        }
        const int4 lk = __ldg(&T.link[nd]);
        const double4 g = ldg4(&T.geo[nd]);
        const int L = lk.w & 0xff;
        const bool leaf = (lk.w >> 8) != 0;
        const unsigned need = (1u << L) - 2u;
        bool pass = false;
        double h2 = 0.0;
        if(valid && (bits & need) == need) {
            double h = hi;
            if(IJ) {
                const double ks = __ldg(&T.ksize[nd]);
                h = hi < ks ? ks : hi;
            }
            h2 = h * h;
            const double l2 = (g.w * 0.5 + h) * (g.w * 0.5 + h);
            const Vec3d d = rij(P, xi, yi, zi, g.x, g.y, g.z);
            double m = d.x * d.x;
            const double m1 = d.y * d.y, m2 = d.z * d.z;
            if(m1 > m) m = m1;
            if(m2 > m) m = m2;
            pass = m <= l2;
        }
        if(leaf) {
            if(pass) {
                for(int q = lk.x; q < lk.y; ++q) {
                    const double4 pq = ldg4(&S.pos[q]);
                    const Vec3d r = rij(P, xi, yi, zi, pq.x, pq.y, pq.z);
                    if(abs2x(r) < h2) {
                        if(cnt < cap) list[row + cnt] = q;
                        ++cnt;
                    }
                }
            }
            nd = lk.z;
        } else {
            bits = pass ? (bits | (1u << L)) : (bits & ~(1u << L));
            nd = __any_sync(FULL_MASK, pass) ? nd + 1 : lk.z;
        }
    }
    return cnt;
}

template <bool IJ>
__global__ void __launch_bounds__(WBLK) k_walk(DevParams P, DevState S, DevTree T, int n, int cap,
                                               int* __restrict__ list, int* __restrict__ count,
                                               DevStatus* __restrict__ st, int guess, double ratio)
{
    const int i = blockIdx.x * WBLK + threadIdx.x;
    const bool valid = i < n;
    double xi = 0, yi = 0, zi = 0, hi = 0;
    if(valid) {
        const double4 p = S.pos[i];
        xi = p.x;
        yi = p.y;
        zi = p.z;
        if(guess) {
            // h guess from the previous density (src/pre_interaction.cpp:61-64)
            constexpr double A = 4.0 * 3.14159265358979323846 / 3.0;
            const double dens = S.thermo[i].x;
            hi = pow(P.nngb * p.w / (dens * A), 1.0 / 3) * ratio;
            S.vel[i].w = hi;
        } else {
            hi = S.vel[i].w;
        }
    }
    const size_t row = (size_t)(valid ? i : 0) * (size_t)cap;
    const int cnt = walk_lanes<IJ>(P, S, T, valid, xi, yi, zi, hi, list, row, cap, st);
    if(valid) {
        count[i] = cnt;
        if(cnt > cap) st->overflow = 1;
        if(cnt > P.nngb * 1000) st->fatal = 1;
        atomicMax(&st->max_count, cnt);
    }
}

// ---------------------------------------------------------------------------
// Group walk.  The set a particle i gets from the reference's recursion is
//   { j : r_ij^2 < h^2  and every box test on the path root -> leaf(j) passes }
// with h = sml_i (gather) or max(sml_i, kernel_size) per node (is_ij).  A box
// test compares the L-infinity distance from x_i to the node centre with
// edge/2 + h.  Particle j lies inside every ancestor's box up to the rounding
// of the node centres (<= ~20 ulp of the coordinate scale), and the test
// radius only grows towards the root, so when r_ij < h_leaf - delta (delta =
// 1e-12 of the domain scale, thousands of ulp) every test on the path passes.
// Only pairs with h_leaf - delta <= r_ij < h_leaf need the reference's tests,
// which are then replayed exactly up the parent chain.
//
// Traversal is therefore done once per warp for the group's bounding box:
// each step the 32 lanes test 32 stack nodes in parallel (a conservative
// superset test), push the children of passing internal nodes (LIFO stack in
// shared memory) and queue passing leaves; queued leaves are tested in
// batches, each lane against its own particle.  A stack overflow marks the
// warp and the host re-runs the call with the per-lane walk.
constexpr int GW_WARPS = 4;
constexpr int GW_STACK = 1024;
constexpr int GW_QUEUE = 64;

__device__ __forceinline__ double interval_gap(double c, double lo, double hi)
{
    return c < lo ? lo - c : (c > hi ? c - hi : 0.0);
}

// exact box test of the reference's recursion at node nd for particle i
template <bool IJ>
__device__ __forceinline__ bool box_pass(const DevParams& P, const DevTree& T, int nd, double xi, double yi, double zi,
                                         double hi)
{
    const double4 g = ldg4(&T.geo[nd]);
    double h = hi;
    if(IJ) {
        const double ks = __ldg(&T.ksize[nd]);
        h = hi < ks ? ks : hi;
    }
    const double l2 = (g.w * 0.5 + h) * (g.w * 0.5 + h);
    const Vec3d d = rij(P, xi, yi, zi, g.x, g.y, g.z);
    double m = d.x * d.x;
    const double m1 = d.y * d.y, m2 = d.z * d.z;
    if(m1 > m) m = m1;
    if(m2 > m) m = m2;
    return m <= l2;
}

template <bool IJ>
__global__ void __launch_bounds__(GW_WARPS * 32) k_walk_group(DevParams P, DevState S, DevTree T, int n, int cap,
                                                             int* __restrict__ list, int* __restrict__ count,
                                                             DevStatus* __restrict__ st, int guess, double ratio)
{
    __shared__ int s_stack[GW_WARPS][GW_STACK];
    __shared__ int s_queue[GW_WARPS][GW_QUEUE];
    __shared__ double4 s_cpos[GW_WARPS][32];
    __shared__ int4 s_clink[GW_WARPS][32];
    __shared__ double s_cks[GW_WARPS][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = (blockIdx.x * GW_WARPS + w) * 32 + lane;
    const bool valid = i < n;
    if(__ballot_sync(FULL_MASK, valid) == 0) return;  // whole warp past the end
    double xi = 0, yi = 0, zi = 0, hi = 0;
    if(valid) {
        const double4 p = S.pos[i];
        xi = p.x;
        yi = p.y;
        zi = p.z;
        if(guess) {
            constexpr double A = 4.0 * 3.14159265358979323846 / 3.0;
            hi = pow(P.nngb * p.w / (S.thermo[i].x * A), 1.0 / 3) * ratio;
            S.vel[i].w = hi;
        } else {
            hi = S.vel[i].w;
        }
    }
    // group bounding box and largest radius
    double lo[3] = {valid ? xi : 1e300, valid ? yi : 1e300, valid ? zi : 1e300};
    double up[3] = {valid ? xi : -1e300, valid ? yi : -1e300, valid ? zi : -1e300};
    double hmax = valid ? hi : 0.0;
    for(int o = 16; o > 0; o >>= 1) {
        for(int k = 0; k < 3; ++k) {
            lo[k] = fmin(lo[k], __shfl_xor_sync(FULL_MASK, lo[k], o));
            up[k] = fmax(up[k], __shfl_xor_sync(FULL_MASK, up[k], o));
        }
        hmax = fmax(hmax, __shfl_xor_sync(FULL_MASK, hmax, o));
    }
    // A window of 32 octree-ordered particles that straddles a large octant
    // boundary has a bounding box far wider than its particles' search
    // spheres; such warps walk per lane instead.
    const double extent = fmax(up[0] - lo[0], fmax(up[1] - lo[1], up[2] - lo[2]));
    if(!(extent <= 4.0 * hmax)) {
        const size_t row0 = (size_t)(valid ? i : 0) * (size_t)cap;
        const int c0 = walk_lanes<IJ>(P, S, T, valid, xi, yi, zi, hi, list, row0, cap, st);
        if(lane == 0) atomicAdd(&st->walk_lane_warps, 1ull);
        if(valid) {
            count[i] = c0;
            if(c0 > cap) st->overflow = 1;
            if(c0 > P.nngb * 1000) st->fatal = 1;
            atomicMax(&st->max_count, c0);
        }
        return;
    }
    if(lane == 0) atomicAdd(&st->walk_group_warps, 1ull);
    // safety margin for the fast acceptance (see above)
    const double4 root = ldg4(&T.geo[0]);
    const double scale = fmax(fabs(root.x), fmax(fabs(root.y), fabs(root.z))) + root.w;
    const double delta = 1e-12 * scale;

    const size_t row = (size_t)(valid ? i : 0) * (size_t)cap;
    int cnt = 0;
    int sp = 0, nq = 0;
    bool overflow = false;
    if(lane == 0) s_stack[w][0] = 0;
    sp = 1;
    __syncwarp();

    auto process = [&](int nproc) {
        // lanes load one queued leaf each, then every lane tests all of them
        const int L = lane < nproc ? s_queue[w][lane] : -1;
        if(L >= 0) {
            const int4 lk = __ldg(&T.link[L]);
            s_clink[w][lane] = make_int4(lk.x, lk.y, L, 0);
            s_cpos[w][lane] = ldg4(&S.pos[lk.x]);
            s_cks[w][lane] = IJ ? __ldg(&T.ksize[L]) : 0.0;
        }
        __syncwarp();
        if(valid) {
            for(int t = 0; t < nproc; ++t) {
                const int4 cl = s_clink[w][t];
                double h = hi;
                if(IJ) {
                    const double ks = s_cks[w][t];
                    h = hi < ks ? ks : hi;
                }
                const double h2 = h * h;
                const double hs = h - delta;
                const double hs2 = hs > 0.0 ? hs * hs : -1.0;
                for(int q = cl.x; q < cl.y; ++q) {
                    const double4 pj = q == cl.x ? s_cpos[w][t] : ldg4(&S.pos[q]);
                    const Vec3d r = rij(P, xi, yi, zi, pj.x, pj.y, pj.z);
                    const double r2 = abs2x(r);
                    if(!(r2 < h2)) continue;
                    bool take = r2 < hs2;
                    if(!take) {
                        // on the radius: replay the reference's box tests up the path
                        take = true;
                        int A = cl.z;
                        for(int up_ = 0; A >= 0 && up_ < 64; ++up_) {
                            if(!box_pass<IJ>(P, T, A, xi, yi, zi, hi)) {
                                take = false;
                                break;
                            }
                            A = A == 0 ? -1 : T.parent[A];
                        }
                    }
                    if(take) {
                        if(cnt < cap) list[row + cnt] = q;
                        ++cnt;
                    }
                }
            }
        }
        __syncwarp();
    };

    const int nnodes = *T.nnodes;
    int steps = 0;
    while(sp > 0) {
        if(++steps > nnodes + 1) {  // each node is pushed at most once
            overflow = true;
            break;
        }
        const int m = sp < 32 ? sp : 32;
        const int nd = lane < m ? s_stack[w][sp - 1 - lane] : -1;
        __syncwarp();
        sp -= m;
        bool pass = false, leaf = false;
        int4 c0 = make_int4(-1, -1, -1, -1), c1 = c0;
        if(nd >= 0) {
            const int4 lk = __ldg(&T.link[nd]);
            const double4 g = ldg4(&T.geo[nd]);
            leaf = (lk.w >> 8) != 0;
            double hh = hmax;
            if(IJ) hh = fmax(hmax, __ldg(&T.ksize[nd]));
            const double reach = (g.w * 0.5 + hh) * (1.0 + 1e-10) + delta;
            const double cc[3] = {g.x, g.y, g.z};
            pass = true;
            for(int k = 0; k < 3; ++k) {
                double gap = interval_gap(cc[k], lo[k], up[k]);
                if(P.periodic) {
                    gap = fmin(gap, interval_gap(cc[k] + P.range[k], lo[k], up[k]));
                    gap = fmin(gap, interval_gap(cc[k] - P.range[k], lo[k], up[k]));
                }
                pass = pass && gap <= reach;
            }
            if(pass && !leaf) {
                const int4* cp = reinterpret_cast<const int4*>(T.child + (size_t)nd * 8);
                c0 = __ldg(cp);
                c1 = __ldg(cp + 1);
            }
        }
        // push children of passing internal nodes (order within a step is free)
        const int kids[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
        int nk = 0;
        for(int k = 0; k < 8; ++k) nk += kids[k] >= 0 ? 1 : 0;
        int incl = nk;
        for(int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(FULL_MASK, incl, o);
            if(lane >= o) incl += u;
        }
        const int total = __shfl_sync(FULL_MASK, incl, 31);
        if(sp + total > GW_STACK) {
            overflow = true;
            break;
        }
        int pos = sp + incl - nk;
        for(int k = 0; k < 8; ++k) {
            if(kids[k] >= 0) s_stack[w][pos++] = kids[k];
        }
        sp += total;
        // queue passing leaves
        const unsigned lb = __ballot_sync(FULL_MASK, pass && leaf);
        if(pass && leaf) s_queue[w][nq + __popc(lb & ((1u << lane) - 1u))] = nd;
        nq += __popc(lb);
        __syncwarp();
        if(nq >= 32) {
            process(32);
            nq -= 32;
            if(lane < nq) s_queue[w][lane] = s_queue[w][32 + lane];
            __syncwarp();
        }
    }
    if(!overflow && nq > 0) process(nq);
    if(overflow) {
        if(lane == 0) st->guard = 2;
        return;
    }
    if(valid) {
        count[i] = cnt;
        if(cnt > cap) st->overflow = 1;
        if(cnt > P.nngb * 1000) st->fatal = 1;
        atomicMax(&st->max_count, cnt);
    }
}

// exhaustive_search (src/exhaustive_search.cpp:11-42): all j with
// r^2 < h_i^2 (gather) or r^2 < max(h_i^2, h_j^2) (is_ij).
__global__ void k_exhaustive(DevParams P, DevState S, int n, int is_ij, int cap, int* __restrict__ list,
                             int* __restrict__ count, DevStatus* __restrict__ st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const double4 p = S.pos[i];
    const double hi = S.vel[i].w;
    const double ki2 = hi * hi;
    int cnt = 0;
    for(int j = 0; j < n; ++j) {
        const double4 pj = S.pos[j];
        const Vec3d r = rij(P, p.x, p.y, p.z, pj.x, pj.y, pj.z);
        const double r2 = abs2x(r);
        double lim = ki2;
        if(is_ij) {
            const double hj = S.vel[j].w;
            const double kj2 = hj * hj;
            lim = ki2 < kj2 ? kj2 : ki2;
        }
        if(r2 < lim) {
            if(cnt < cap) list[(size_t)i * cap + cnt] = j;
            ++cnt;
        }
    }
    count[i] = cnt;
    if(cnt > cap) st->overflow = 1;
    if(cnt > P.nngb * 1000) st->fatal = 1;
    atomicMax(&st->max_count, cnt);
}

__global__ void k_counts_by_id(int n, const int* __restrict__ id, const int* __restrict__ count,
                               unsigned long long* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) out[id[i]] = (unsigned long long)count[i];
}

__global__ void k_fill_by_id(int n, int cap, const int* __restrict__ id, const int* __restrict__ count,
                             const int* __restrict__ list, const unsigned long long* __restrict__ off,
                             int* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const unsigned long long b = off[id[i]];
    const int c = count[i];
    for(int k = 0; k < c; ++k) out[b + k] = id[list[(size_t)i * cap + k]];
}

int run_walk(sphgpu_ctx* c, int which, bool guess, double ratio, bool exhaustive, int is_ij, int* launches)
{
    cudaStream_t st = c->stream;
    const int n = c->n;
    bool per_lane = false;
    for(int attempt = 0; attempt < 6; ++attempt) {
        ++*launches;
        const int64_t cap = which == 0 ? c->gcap : c->pcap;
        int* list = which == 0 ? c->d_glist : c->d_plist;
        int* count = which == 0 ? c->d_gcount : c->d_pcount;
        SPHGPU_CUDA(c, cudaMemsetAsync(c->d_status, 0, 3 * sizeof(int), st));
        SPHGPU_CUDA(c, cudaMemsetAsync(&c->d_status->guard, 0, sizeof(int), st));
        if(exhaustive) {
            k_exhaustive<<<grid_for(n, 128), 128, 0, st>>>(c->dp, c->s, n, is_ij, (int)cap, list, count, c->d_status);
        } else if(c->walk_mode == 0 && !per_lane) {
            const unsigned grid = grid_for(n, GW_WARPS * 32);
            if(which == 0) {
                k_walk_group<false><<<grid, GW_WARPS * 32, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                                   c->d_status, guess ? 1 : 0, ratio);
            } else {
                k_walk_group<true><<<grid, GW_WARPS * 32, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                                  c->d_status, 0, 1.0);
            }
        } else if(which == 0) {
            k_walk<false><<<grid_for(n, WBLK), WBLK, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                            c->d_status, guess ? 1 : 0, ratio);
        } else {
            k_walk<true><<<grid_for(n, WBLK), WBLK, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                           c->d_status, 0, 1.0);
        }
        SPHGPU_LAUNCH_CHECK(c, "neighbour walk");
        SPHGPU_CUDA(c, cudaMemcpyAsync(&c->h_status, c->d_status, 5 * sizeof(int), cudaMemcpyDeviceToHost, st));
        SPHGPU_CUDA(c, cudaStreamSynchronize(st));
        if(c->h_status.fatal) {
            return fail(c, SPHGPU_ERR_NEIGHBOR_OVERFLOW,
                        "Neighbor list overflow: more than neighborNumber * 1000 neighbours");
        }
        if(c->h_status.guard == 2 && !per_lane) {
            // a warp's traversal stack overflowed: redo this call with the per-lane walk
            per_lane = true;
            ++c->walk_fallbacks;
            continue;
        }
        if(c->h_status.guard) return fail(c, SPHGPU_ERR_STATE, "tree walk exceeded the node count (corrupt tree)");
        if(which == 0) c->max_gather = c->h_status.max_count;
        else c->max_pair = c->h_status.max_count;
        if(!c->h_status.overflow) return attempt == 0 ? SPHGPU_OK : SPHGPU_RETRIED;
        // grow to the largest list seen (+12.5%, rounded to 32) and re-run;
        // a guessed h is recomputed identically on the re-run
        int64_t want = c->h_status.max_count + c->h_status.max_count / 8;
        want = (want + 31) / 32 * 32;
        const int rc = ensure_list_capacity(c, which, want);
        if(rc < 0) return rc;
        ++c->retries;
    }
    return fail(c, SPHGPU_ERR_NEIGHBOR_OVERFLOW, "neighbour list capacity did not converge");
}

}  // namespace

int gather_walk(sphgpu_ctx* c, bool compute_guess, double ratio)
{
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "neighbour search before tree make");
    stage_begin(c, SPHGPU_T_GATHER_WALK);
    int launches = 0;
    const int rc = run_walk(c, 0, compute_guess, ratio, false, 0, &launches);
    stage_end(c, SPHGPU_T_GATHER_WALK, launches);
    return rc;
}

int pair_walk(sphgpu_ctx* c)
{
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "neighbour search before tree make");
    stage_begin(c, SPHGPU_T_PAIR_WALK);
    int launches = 0;
    const int rc = run_walk(c, 1, false, 1.0, false, 1, &launches);
    stage_end(c, SPHGPU_T_PAIR_WALK, launches);
    return rc;
}

// Copy list `which` (0 gather, 1 pair) to a host CSR in caller order with
// caller ids.
int export_lists(sphgpu_ctx* c, int which, int64_t* offsets, int32_t* ids, int64_t cap)
{
    cudaStream_t st = c->stream;
    const int n = c->n;
    const int64_t lcap = which == 0 ? c->gcap : c->pcap;
    const int* list = which == 0 ? c->d_glist : c->d_plist;
    const int* count = which == 0 ? c->d_gcount : c->d_pcount;
    unsigned long long *d_cnt = nullptr, *d_off = nullptr, *d_tot = nullptr;
    SPHGPU_CUDA(c, cudaMallocAsync(&d_cnt, sizeof(unsigned long long) * (size_t)(2 * n + 2), st));
    d_off = d_cnt + n;
    d_tot = d_off + n;
    k_counts_by_id<<<grid_for(n, 256), 256, 0, st>>>(n, c->s.id, count, d_cnt);
    exclusive_scan(d_cnt, d_off, n, d_tot, c->scan, st);
    unsigned long long total = 0;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&total, d_tot, sizeof(total), cudaMemcpyDeviceToHost, st));
    std::vector<unsigned long long> off(n);
    SPHGPU_CUDA(c, cudaMemcpyAsync(off.data(), d_off, sizeof(unsigned long long) * (size_t)n,
                                   cudaMemcpyDeviceToHost, st));
    SPHGPU_CUDA(c, cudaStreamSynchronize(st));
    for(int i = 0; i < n; ++i) offsets[i] = (int64_t)off[i];
    offsets[n] = (int64_t)total;
    int rc = SPHGPU_OK;
    if(ids) {
        if((int64_t)total > cap) {
            rc = fail(c, SPHGPU_ERR_ARG, "neighbour id buffer too small");
        } else {
            int* d_ids = nullptr;
            SPHGPU_CUDA(c, cudaMallocAsync(&d_ids, sizeof(int) * (size_t)(total + 1), st));
            k_fill_by_id<<<grid_for(n, 256), 256, 0, st>>>(n, (int)lcap, c->s.id, count, list, d_off, d_ids);
            SPHGPU_CUDA(c, cudaMemcpyAsync(ids, d_ids, sizeof(int) * (size_t)total, cudaMemcpyDeviceToHost, st));
            SPHGPU_CUDA(c, cudaFreeAsync(d_ids, st));
        }
    }
    SPHGPU_CUDA(c, cudaFreeAsync(d_cnt, st));
    SPHGPU_CUDA(c, cudaStreamSynchronize(st));
    return rc;
}

int exhaustive_lists(sphgpu_ctx* c, int is_ij, int64_t* offsets, int32_t* ids, int64_t cap)
{
    int launches = 0;
    const int rc = run_walk(c, 1, false, 1.0, true, is_ij, &launches);
    c->launches += launches;
    if(rc < 0) return rc;
    return export_lists(c, 1, offsets, ids, cap);
}

}  // namespace sphgpu
