// gravity_mixed.cu — GravityForce::calculation, mixed-precision form.
//
// Reference: src/gravity_force.cpp:52-89, BHNode::calc_force
// (src/bhtree.cpp:347-393), softening kernels src/bhtree.cpp:318-345.
//
// The same per-lane stackless preorder walk as the FP64 form (gravity.cu): a
// lane accepts its node as a monopole and jumps over the subtree, or opens it
// (a leaf is summed pairwise with spline softening, an internal node is
// descended into).  What changes:
// * node records of 32 bytes, one sector per node (two 16-byte loads per
//   node test instead of the FP64 form's three from three arrays; the walk
//   is bound by L1 requests, 89 % of the L1 throughput on the Evrard sphere
//   at 1.1 M with three loads; both halves now come in one 256-bit access:
//   59.5 -> 56.7 ms per step on the 8.78 M sphere):
//   a = {com_hi, G m} in FP32, b = {com_lo in bf16, leaf flag, skip, edge^2},
//   where com_hi = (float)com and com_lo = com - com_hi: the offset
//   x_i - com = (x_hi - com_hi) + (x_lo - com_lo) keeps about 32 bits of the
//   FP64 position.  A leaf's particle range is read only when it is opened;
// * opening test, monopole and softened pair terms in FP32 (FMA contraction
//   allowed in this file);
// * FP32 accumulation of the terms, folded into the particle's FP64
//   acceleration and potential every 32 nodes and at the end of the walk.
// The form is held to the FP64 form by tolerance, not bit for bit.
// Measured alternatives on the same sphere: a warp-synchronous walk (cursor =
// the warp's smallest next node, broadcast loads) 9.96 ms vs 9.30 ms per-lane
// with three loads; walks shared by 2, 4, 8, 16 lanes 17.6 / 14.2 / 12.3 /
// 11.3 ms; queueing opened leaves for warp-wide pair batches 9.65 ms.  With
// the present records and pair terms (6.31 ms): lanes that take the next
// particle of a per-warp range when their walk ends, instead of waiting for
// the warp's longest walk, 10.07 ms (the lanes' walks drift apart and lose
// the L1 reuse of walking neighbouring particles in step).  Running this walk
// on a second stream beside the symmetric walk and the force of the step
// (Evrard 8.8 M): 166.5 ms per step against 157 ms one after the other; the
// kernels slow each other down (force 17 -> 82 ms, gravity 55 -> 88 ms).
// Loading the next node's record as soon as the opening test has chosen it
// (which helps the FP64 walk a little): 56.6 -> 59.6 ms.
// The records are rebuilt from the tree on every call (one streaming pass over
// the nodes), so they always match the current tree.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int MBLK = 128;
constexpr int FOLD = 32;  // nodes between folds of the FP32 partial sums

__device__ __forceinline__ unsigned bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

// Node records, 32 bytes per node (one sector): a = {com_hi x, y, z, G m};
// b = {bf16 com_lo x | y << 16, bf16 com_lo z | leaf << 16, skip, edge^2
// (float bits)}.
struct __align__(32) GNode {
    float4 a;
    int4 b;
};

__global__ void k_gnode(DevTree Tr, double G, GNode* __restrict__ rec, int cap)
{
    const int nn = min(*Tr.nnodes, cap);
    const double root_edge = Tr.geo[0].w;
    for(int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < nn; nd += gridDim.x * blockDim.x) {
        const double4 mc = Tr.mass[nd];
        const int4 lk = Tr.link[nd];
        const double edge = ldexp(root_edge, 1 - (lk.w & 0xff));
        const float hx = (float)mc.x, hy = (float)mc.y, hz = (float)mc.z;
        rec[nd].a = make_float4(hx, hy, hz, (float)(G * mc.w));
        const unsigned lx = bf16_bits((float)(mc.x - (double)hx)), ly = bf16_bits((float)(mc.y - (double)hy));
        const unsigned lz = bf16_bits((float)(mc.z - (double)hz));
        const unsigned leaf = (lk.w >> 8) != 0 ? 1u : 0u;
        rec[nd].b = make_int4((int)(lx | (ly << 16)), (int)(lz | (leaf << 16)), lk.z, __float_as_int((float)(edge * edge)));
    }
}

// Spline softening of one pair in FP32: the kernels f (potential) and g (force
// / r) of the Hernquist & Katz spline (src/bhtree.cpp:318-345) for one smoothing length,
// with their divisions by e = h / 2 and by r turned into products with the
// reciprocals einv = 1 / e and rinv = 1 / r.
__device__ __forceinline__ void hk_fg(float r, float rinv, float einv, float& f, float& g)
{
    const float u = r * einv;
    const float u2 = u * u;
    if(u < 1.f) {
        f = (-0.5f * u2 * (1.f / 3.f - 0.15f * u2 + u2 * u * 0.05f) + 1.4f) * einv;
        g = (4.f / 3.f - 1.2f * u2 + 0.5f * u2 * u) * (einv * einv * einv);
    } else if(u < 2.f) {
        const float u3 = u2 * u;
        f = -(1.f / 15.f) * rinv + (-u2 * (4.f / 3.f - u + 0.3f * u2 - u3 * (1.f / 30.f)) + 1.6f) * einv;
        g = (-1.f / 15.f + 8.f / 3.f * u3 - 3.f * u3 * u + 1.2f * u3 * u2 - u3 * u3 * (1.f / 6.f)) *
            (rinv * rinv * rinv);
    } else {
        f = rinv;
        g = rinv * rinv * rinv;
    }
}

// Minimum image of an FP32 offset (include/periodic.hpp:34-72): the closest of
// d, d + L, d - L.
__device__ __forceinline__ float min_image_f(float d, float L)
{
    if(fabsf(d) <= 0.5f * L) return d;
    const float b = d + L, c = d - L;
    const float ad = fabsf(d), ab = fabsf(b), ac = fabsf(c);
    if(ad <= ab && ad <= ac) return d;
    if(ab <= ac) return b;
    return c;
}

__global__ void __launch_bounds__(MBLK, 8) k_gravity_mixed(DevParams P, DevState S, DevTree Tr,
                                                        const GNode* __restrict__ rec, int n,
                                                        DevStatus* __restrict__ st, float* __restrict__ accabs)
{
    const int i = blockIdx.x * MBLK + threadIdx.x;
    const bool valid = i < n;
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
    const float xh = (float)xi, yh = (float)yi, zh = (float)zi;
    const float xl = (float)(xi - (double)xh), yl = (float)(yi - (double)yh), zl = (float)(zi - (double)zh);
    const float einv_i = (float)(2.0 / hi);  // 1 / e, e = h / 2
    const float theta2 = (float)P.theta2;
    const float Gf = (float)P.G;
    const bool per = P.periodic;
    const float Lx = (float)P.range[0], Ly = (float)P.range[1], Lz = (float)P.range[2];
    double ax = acc.x, ay = acc.y, az = acc.z, phi = 0.0;
    float fx = 0.f, fy = 0.f, fz = 0.f, fp = 0.f;
    float gabs = 0.f;  // sum of |FP32 terms|, the rounding-error scale of the acceleration
    int since = 0;
    const int nnodes = *Tr.nnodes;
    int nd = valid ? 0 : nnodes, steps = 0;
    unsigned n_mono = 0, n_leaf = 0;  // work counters of this lane (steps = nodes met)
    while(nd < nnodes) {
        if(++steps > nnodes) {  // corrupt node table: report, never loop
            atomicOr(&st->pass_guard, PASS_GUARD_GRAVITY32);
            break;
        }
        float4 a;
        int4 b;
        // the 32-byte record in one 256-bit access
        asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
            : "l"(rec + nd));
        const bool leaf = (b.y >> 16) & 1;
        const float l2 = __int_as_float(b.w);
        float dx = (xh - a.x) + (xl - __uint_as_float((unsigned)b.x << 16));
        float dy = (yh - a.y) + (yl - __uint_as_float((unsigned)b.x & 0xffff0000u));
        float dz = (zh - a.z) + (zl - __uint_as_float((unsigned)b.y << 16));
        if(per) {
            dx = min_image_f(dx, Lx);
            dy = min_image_f(dy, Ly);
            dz = min_image_f(dz, Lz);
        }
        const float d2 = dx * dx + dy * dy + dz * dz;
        const bool open = (l2 > theta2 * d2) || (d2 < l2);
        if(!open) {
            ++n_mono;
            const float rinv = rsqrtf(d2);
            const float gr = a.w * rinv;
            const float s = gr * rinv * rinv;
            fp -= gr;
            fx -= dx * s;
            fy -= dy * s;
            fz -= dz * s;
            gabs += s * (fabsf(dx) + fabsf(dy) + fabsf(dz));
        } else if(leaf) {
            const int4 lk = __ldg(&Tr.link[nd]);
            n_leaf += (unsigned)(lk.y - lk.x) - ((i >= lk.x && i < lk.y) ? 1u : 0u);
            for(int q = lk.x; q < lk.y; ++q) {
                if(q == i) continue;
                const double4 pq = ldg4(&S.pos[q]);
                const float hq = (float)__ldg(&S.vel[q].w);
                const Vec3d r = rij(P, xi, yi, zi, pq.x, pq.y, pq.z);
                const float rx = (float)r.x, ry = (float)r.y, rz = (float)r.z;
                const float r2 = rx * rx + ry * ry + rz * rz;
                const float rinv = rsqrtf(r2);
                const float rr = r2 * rinv;
                float f1, g1, f2, g2;
                hk_fg(rr, rinv, einv_i, f1, g1);
                hk_fg(rr, rinv, __fdividef(2.f, hq), f2, g2);
                const float gm = Gf * (float)pq.w;
                fp -= gm * (f1 + f2) * 0.5f;
                const float c = gm * (g1 + g2) * 0.5f;
                fx -= rx * c;
                fy -= ry * c;
                fz -= rz * c;
                gabs += fabsf(c) * (fabsf(rx) + fabsf(ry) + fabsf(rz));
            }
        }
        if(++since == FOLD) {
            ax += (double)fx;
            ay += (double)fy;
            az += (double)fz;
            phi += (double)fp;
            fx = fy = fz = fp = 0.f;
            since = 0;
        }
        nd = (open && !leaf) ? nd + 1 : b.z;
    }
    if(valid) {
        S.acc[i] = make_double4(ax + (double)fx, ay + (double)fy, az + (double)fz, acc.w);
        S.visc[i].w = phi + (double)fp;
        if(accabs) accabs[i] += gabs;
    }
    block_count(&st->grav_nodes, (unsigned)min(steps, nnodes));
    block_count(&st->grav_mono, n_mono);
    block_count(&st->grav_leaf_pairs, n_leaf);
}

}  // namespace

int gravity_nodes_mixed(sphgpu_ctx* c)
{
    if(c->gnode_cap < c->node_cap) {
        if(c->d_gnode) cudaFree(c->d_gnode);
        c->d_gnode = nullptr;
        c->gnode_cap = 0;
        SPHGPU_CUDA(c, cudaMalloc(&c->d_gnode, sizeof(GNode) * (size_t)c->node_cap));
        c->gnode_cap = c->node_cap;
    }
    k_gnode<<<148 * 8, 256, 0, c->stream>>>(c->t, c->dp.G, static_cast<GNode*>(c->d_gnode), c->gnode_cap);
    return SPHGPU_OK;
}

int gravity_walk_mixed(sphgpu_ctx* c)
{
    if(c->gnode_cap < c->node_cap) return fail(c, SPHGPU_ERR_STATE, "mixed gravity walk before its node records");
    k_gravity_mixed<<<grid_for(c->n, MBLK), MBLK, 0, c->stream>>>(
        c->dp, c->s, c->t, static_cast<const GNode*>(c->d_gnode), c->n, c->d_status, c->d_accabs);
    return SPHGPU_OK;
}

}  // namespace sphgpu
