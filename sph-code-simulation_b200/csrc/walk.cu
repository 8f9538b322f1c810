// walk.cu — batched BHTree::neighbor_search and exhaustive_search.
//
// Reference: BHNode::neighbor_search (src/bhtree.cpp:277-316) — per node, the
// L-infinity box test |d_k| <= edge/2 + h against the node centre, then at a
// leaf the radius test r^2 < h^2 on every particle of the leaf list, with
// h = sml (gather) or max(sml, node.kernel_size) (is_ij).
//
// Two walks produce the same sets.
//
// Group walk (default, k_walk_group): a warp owns 32 consecutive particles in
// octree order.  The warp traverses the tree once for the bounding box of its
// particles (a conservative superset test, 32 nodes per step from a shared
// memory stack), queues passing leaves, and queues whole nodes that are small
// or lie inside the search box instead of descending into them.  Queued
// particles are staged 32 at a time; every lane classifies them against its
// own particle in FP32 with rigorously rounded thresholds (certainly inside /
// certainly outside / a thin band at the radius), and only band pairs run the
// reference's FP64 test, with the box tests replayed up the parent chain for
// pairs on the radius.  Warps whose particles straddle a large octant
// boundary are split into compact sub-groups walked one after another.
//
// Per-lane walk (k_walk, the fallback and cross-check): each lane keeps one
// bit per tree level: bit L says "my box test passed at the current level-L
// ancestor".  A node at level L is live for a lane iff bits 1..L-1 are all
// set: exactly the set of nodes the reference's recursion would visit for
// that particle.  The warp descends into a node (index + 1) when any live lane
// passes, else jumps over the subtree (skip pointer).  Every test is evaluated
// in unfused FP64 (this file builds with -fmad=false), so each lane's list
// equals the reference's list as a set, and even in order before the
// reference's distance sort.
//
// Lists go to an ELL buffer (capacity slots per particle, row-major).  A list
// longer than the capacity is counted but not stored; the host grows the
// buffer and re-runs (status.overflow).  More than neighbor_number * 1000
// entries is the reference's fatal overflow (src/bhtree.cpp:129-135).
#include <algorithm>
#include <cmath>
#include <cstddef>
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

// Skin (Verlet) gather lists: the gather walk runs with radius factor x the
// guessed radius and records each particle's walk radius and position, so
// later steps can reuse the lists while every particle's true gather sphere
// stays inside its skin sphere (skin_check).  factor = 1, r = x = null: the
// reference's exact lists.
struct SkinOut {
    double factor;
    double* r;
    double4* x;
};

template <bool IJ>
__global__ void __launch_bounds__(WBLK) k_walk(DevParams P, DevState S, DevTree T, int n, int cap,
                                               int* __restrict__ list, int* __restrict__ count,
                                               DevStatus* __restrict__ st, int guess, double ratio, SkinOut sk)
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
            const double g = pow(P.nngb * p.w / (dens * A), 1.0 / 3) * ratio;
            S.vel[i].w = g;
            hi = g * sk.factor;
            if(sk.r) {
                sk.r[i] = hi;
                sk.x[i] = p;
            }
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
// Traversal is therefore done once per (sub-)group for its bounding box:
// each step the 32 lanes test 32 stack nodes in parallel (a conservative
// superset test), push the children of passing internal nodes (LIFO stack in
// shared memory) and queue passing leaves and whole nodes; queued particles
// are classified in chunks of 32, each lane against its own particle.  Any
// superset of the reference's candidates gives the same lists, because the
// per-pair classification alone decides membership.  A stack overflow marks
// the warp and the host re-runs the call with the per-lane walk.
constexpr int GW_WARPS = 2;  // warps per block (2: 1 M shear walk 4.38 -> 4.14 ms against 4; 1: 4.33)
constexpr int GW_STACK = 1024;
constexpr int GW_QUEUE = 64;
constexpr int GW_WHOLE = 8;   // nodes with at most this many particles are queued whole
constexpr double GW_SPLIT = 6.0;  // sub-group extent limit, in units of its largest radius

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
                                                             DevStatus* __restrict__ st, int guess, double ratio,
                                                             SkinOut sk)
{
    __shared__ int s_stack[GW_WARPS][GW_STACK];
    __shared__ int s_queue[GW_WARPS][GW_QUEUE];
    __shared__ float4 s_cf[GW_WARPS][32];
    __shared__ double4 s_cpos[GW_WARPS][32];
    __shared__ int s_cid[GW_WARPS][32];
    __shared__ float s_ctin[GW_WARPS][32];
    __shared__ int s_loff[GW_WARPS][32];
    __shared__ int s_lstart[GW_WARPS][32];
    __shared__ double s_box[GW_WARPS][32][7];
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
            const double g = pow(P.nngb * p.w / (S.thermo[i].x * A), 1.0 / 3) * ratio;
            S.vel[i].w = g;
            hi = g * sk.factor;
            if(sk.r) {
                sk.r[i] = hi;
                sk.x[i] = p;
            }
        } else {
            hi = S.vel[i].w;
        }
    }
    // Sub-groups.  A window of 32 octree-ordered particles that straddles a
    // large octant boundary has a bounding box far wider than its particles'
    // search spheres.  The warp is split into aligned sub-groups of s lanes
    // (s = 32, 16, ..., 1: the largest s for which every sub-group's extent
    // is at most GW_SPLIT times its largest radius) and the cooperative walk
    // runs once per sub-group, all lanes traversing and staging, only the
    // sub-group's lanes testing candidates.
    const double own_lo[3] = {valid ? xi : 1e300, valid ? yi : 1e300, valid ? zi : 1e300};
    const double own_up[3] = {valid ? xi : -1e300, valid ? yi : -1e300, valid ? zi : -1e300};
    const double own_h = valid ? hi : 0.0;
    int s = 1;
    {
        double l[3] = {own_lo[0], own_lo[1], own_lo[2]}, u[3] = {own_up[0], own_up[1], own_up[2]}, hm = own_h;
        for(int o = 1; o < 32; o <<= 1) {
            for(int k = 0; k < 3; ++k) {
                l[k] = fmin(l[k], __shfl_xor_sync(FULL_MASK, l[k], o));
                u[k] = fmax(u[k], __shfl_xor_sync(FULL_MASK, u[k], o));
            }
            hm = fmax(hm, __shfl_xor_sync(FULL_MASK, hm, o));
            const double e = fmax(u[0] - l[0], fmax(u[1] - l[1], u[2] - l[2]));
            if(__all_sync(FULL_MASK, e <= GW_SPLIT * hm)) s = 2 * o;
        }
    }
    {
        // each sub-group's box and radius, kept in shared memory
        double lo[3] = {own_lo[0], own_lo[1], own_lo[2]}, up[3] = {own_up[0], own_up[1], own_up[2]};
        double hmax = own_h;
        for(int o = 1; o < s; o <<= 1) {
            for(int k = 0; k < 3; ++k) {
                lo[k] = fmin(lo[k], __shfl_xor_sync(FULL_MASK, lo[k], o));
                up[k] = fmax(up[k], __shfl_xor_sync(FULL_MASK, up[k], o));
            }
            hmax = fmax(hmax, __shfl_xor_sync(FULL_MASK, hmax, o));
        }
        if(lane % s == 0) {
            double* b = s_box[w][lane / s];
            b[0] = lo[0], b[1] = lo[1], b[2] = lo[2], b[3] = up[0], b[4] = up[1], b[5] = up[2], b[6] = hmax;
        }
        __syncwarp();
    }
    if(lane == 0) atomicAdd(s == 32 ? &st->walk_group_warps : &st->walk_split_warps, 1ull);
    // safety margin for the fast acceptance (see above)
    const double4 root = ldg4(&T.geo[0]);
    const double scale = fmax(fabs(root.x), fmax(fabs(root.y), fabs(root.z))) + root.w;
    const double delta = 1e-12 * scale;

    const size_t row = (size_t)(valid ? i : 0) * (size_t)cap;
    int cnt = 0;
    bool overflow = false;
    for(int sg = 0; sg < 32 / s && !overflow; ++sg) {
        const bool act = valid && lane / s == sg;
        if(__ballot_sync(FULL_MASK, act) == 0) continue;
        const double* bb = s_box[w][sg];
        const double blo[3] = {bb[0], bb[1], bb[2]}, bup[3] = {bb[3], bb[4], bb[5]};
        const double bh = bb[6];
        const double bext = fmax(bup[0] - blo[0], fmax(bup[1] - blo[1], bup[2] - blo[2]));
        int sp = 0, nq = 0;
        if(lane == 0) s_stack[w][0] = 0;
        sp = 1;
        __syncwarp();

        // FP32 classification.  Candidates are staged once per warp as FP32
        // offsets b_j = x_j - c from the group centre c (minimum image applied
        // once, in FP64); each lane holds a_i = x_i - c.  For any candidate that
        // can matter (|a_i - b_j| <~ h) the FP32 distance |a_i - b_j| differs from
        // the exact r by at most E = 2^-22 ext + 2^-21 h (conversions and the
        // subtraction; ext = sub-group extent) and the FP32 sum of squares r2f from
        // |a_i - b_j|^2 by a factor 1 +- 3 * 2^-24.  Hence
        //   r2f >= Tout(h) = ((1 + 2^-20) h + 2^-21 ext)^2 (1 + 2^-20)  =>  r >= h,
        //   r2f <  Tin(h)  = ((1 - 2^-20) (h - delta - E))^2 (1 - 2^-20) =>  r < h - delta,
        // both thresholds rounded outwards to FP32.  A pair below Tin is in the
        // reference's set with every box test on its path passing (see above),
        // so it is taken without FP64 work; only pairs between the thresholds run
        // the exact FP64 test.  With periodic wrapping the FP32 offset is the
        // minimum image only if |b_j| + ext/2 < L/2 on every axis (|a_i| <= ext/2);
        // other candidates are staged with NaN offsets and always run the exact
        // test.  Each lane classifies a chunk of 32 staged candidates branch-free
        // into two bit masks (inside, band), runs the exact test for the band
        // bits and writes the taken candidates in chunk order.
        const double cx = 0.5 * (blo[0] + bup[0]), cy = 0.5 * (blo[1] + bup[1]), cz = 0.5 * (blo[2] + bup[2]);
        const double ext_x = bup[0] - blo[0], ext_y = bup[1] - blo[1], ext_z = bup[2] - blo[2];
        const float ax = (float)(xi - cx), ay = (float)(yi - cy), az = (float)(zi - cz);
        auto t_out = [&](double h) -> float {
            const double t = h * (1.0 + 0x1p-20) + 0x1p-21 * bext;
            return __double2float_ru(t * t * (1.0 + 0x1p-20));
        };
        auto t_in = [&](double h) -> float {
            const double t = (h - delta - (0x1p-22 * bext + 0x1p-21 * h)) * (1.0 - 0x1p-20);
            return t > 0.0 ? __double2float_rd(t * t * (1.0 - 0x1p-20)) : -1.0f;
        };
        const float Ti_out = act ? t_out(hi) : -1.0f;
        const float Ti_in = act ? t_in(hi) : -1.0f;
        const float F_INF = __int_as_float(0x7f800000);
        const float F_NAN = __int_as_float(0x7fffffff);

        auto process = [&](int nproc) {
            // expand the queued nodes into their particles (warp prefix sum)
            int lstart = 0, lcnt = 0;
            if(lane < nproc) {
                const int4 lk = __ldg(&T.link[s_queue[w][lane]]);
                lstart = lk.x;
                lcnt = lk.y - lk.x;
            }
            int incl = lcnt;
            for(int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(FULL_MASK, incl, o);
                if(lane >= o) incl += u;
            }
            const int total = __shfl_sync(FULL_MASK, incl, 31);
            s_loff[w][lane] = incl - lcnt;
            s_lstart[w][lane] = lstart;
            __syncwarp();
            for(int base = 0; base < total; base += 32) {
                const int g = base + lane;
                if(g < total) {
                    // the leaf holding candidate g: largest t < nproc with loff[t] <= g
                    int t = 0;
                    for(int s = 16; s > 0; s >>= 1) {
                        if(t + s < nproc && s_loff[w][t + s] <= g) t += s;
                    }
                    const int q = s_lstart[w][t] + (g - s_loff[w][t]);
                    const double4 pj = ldg4(&S.pos[q]);
                    const double ks = IJ ? __ldg(&T.pks[q]) : 0.0;
                    double bx = xsub(pj.x, cx), by = xsub(pj.y, cy), bz = xsub(pj.z, cz);
                    bool pre = true;
                    if(P.periodic) {
                        bx = min_image(bx, P.range[0]);
                        by = min_image(by, P.range[1]);
                        bz = min_image(bz, P.range[2]);
                        pre = fabs(bx) + 0.5 * ext_x < 0.499999 * P.range[0]
                            && fabs(by) + 0.5 * ext_y < 0.499999 * P.range[1]
                            && fabs(bz) + 0.5 * ext_z < 0.499999 * P.range[2];
                    }
                    float tko = -1.0f, tki = -1.0f;
                    if(IJ) {
                        tko = t_out(ks);
                        tki = t_in(ks);
                    }
                    float fx = (float)bx, fy = (float)by, fz = (float)bz;
                    if(!pre) fx = fy = fz = F_NAN;  // classified as band: exact test
                    s_cf[w][lane] = make_float4(fx, fy, fz, tko);
                    s_ctin[w][lane] = tki;
                    s_cpos[w][lane] = make_double4(pj.x, pj.y, pj.z, ks);
                    s_cid[w][lane] = q;
                } else {
                    // padding: infinitely far, never taken
                    s_cf[w][lane] = make_float4(F_INF, F_INF, F_INF, -1.0f);
                    s_ctin[w][lane] = -1.0f;
                }
                __syncwarp();
                if(act) {
                    unsigned in_mask = 0u, band_mask = 0u;
    #pragma unroll
                    for(int k = 0; k < 32; ++k) {
                        const float4 b = s_cf[w][k];
                        const float dx = ax - b.x, dy = ay - b.y, dz = az - b.z;
                        const float r2f = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        const float to = IJ ? fmaxf(Ti_out, b.w) : Ti_out;
                        const float ti = IJ ? fmaxf(Ti_in, s_ctin[w][k]) : Ti_in;
                        const bool inside = r2f < ti;
                        const bool band = !inside && !(r2f >= to);  // NaN offsets land here
                        in_mask |= (unsigned)inside << k;
                        band_mask |= (unsigned)band << k;
                    }
                    while(band_mask) {
                        const int k = __ffs(band_mask) - 1;
                        band_mask &= band_mask - 1u;
                        const int q = s_cid[w][k];
                        const double4 pj = s_cpos[w][k];
                        double h = hi;
                        if(IJ) h = hi < pj.w ? pj.w : hi;
                        const Vec3d r = rij(P, xi, yi, zi, pj.x, pj.y, pj.z);
                        const double r2 = abs2x(r);
                        if(!(r2 < h * h)) continue;
                        const double hs = h - delta;
                        bool take = hs > 0.0 && r2 < hs * hs;
                        if(!take) {
                            // on the radius: replay the reference's box tests up the path
                            take = true;
                            int A = __ldg(&T.leaf_of[q]);
                            for(int up_ = 0; A >= 0 && up_ < 64; ++up_) {
                                if(!box_pass<IJ>(P, T, A, xi, yi, zi, hi)) {
                                    take = false;
                                    break;
                                }
                                A = A == 0 ? -1 : T.parent[A];
                            }
                        }
                        if(take) in_mask |= 1u << k;
                    }
                    while(in_mask) {
                        const int k = __ffs(in_mask) - 1;
                        in_mask &= in_mask - 1u;
                        if(cnt < cap) list[row + cnt] = s_cid[w][k];
                        ++cnt;
                    }
                }
                __syncwarp();
            }
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
                double hh = bh;
                if(IJ) hh = fmax(bh, __ldg(&T.ksize[nd]));
                const double reach = (g.w * 0.5 + hh) * (1.0 + 1e-10) + delta;
                const double cc[3] = {g.x, g.y, g.z};
                pass = true;
                for(int k = 0; k < 3; ++k) {
                    double gap = interval_gap(cc[k], blo[k], bup[k]);
                    if(P.periodic) {
                        gap = fmin(gap, interval_gap(cc[k] + P.range[k], blo[k], bup[k]));
                        gap = fmin(gap, interval_gap(cc[k] - P.range[k], blo[k], bup[k]));
                    }
                    pass = pass && gap <= reach;
                }
                if(pass && !leaf) {
                    // queue every particle of a small node, or of a node whose
                    // box lies inside the group's search box (all its leaves
                    // would pass), instead of descending: the candidate set only
                    // grows, and the per-pair classification decides
                    bool whole = lk.y - lk.x <= GW_WHOLE;
                    if(!whole) {
                        const double he = g.w * 0.5;
                        whole = true;
                        for(int k = 0; k < 3; ++k) whole = whole && cc[k] - he >= blo[k] - bh && cc[k] + he <= bup[k] + bh;
                    }
                    if(whole) {
                        leaf = true;
                    } else {
                        const int4* cp = reinterpret_cast<const int4*>(T.child + (size_t)nd * 8);
                        c0 = __ldg(cp);
                        c1 = __ldg(cp + 1);
                    }
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
    }
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

int run_walk(sphgpu_ctx* c, int which, bool guess, double ratio, bool exhaustive, int is_ij, int* launches,
             SkinOut sk = SkinOut{1.0, nullptr, nullptr})
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
                                                                   c->d_status, guess ? 1 : 0, ratio, sk);
            } else {
                k_walk_group<true><<<grid, GW_WARPS * 32, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                                  c->d_status, 0, 1.0, SkinOut{1.0, nullptr, nullptr});
            }
        } else if(which == 0) {
            k_walk<false><<<grid_for(n, WBLK), WBLK, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                            c->d_status, guess ? 1 : 0, ratio, sk);
        } else {
            k_walk<true><<<grid_for(n, WBLK), WBLK, 0, st>>>(c->dp, c->s, c->t, n, (int)cap, list, count,
                                                           c->d_status, 0, 1.0, SkinOut{1.0, nullptr, nullptr});
        }
        SPHGPU_LAUNCH_CHECK(c, "neighbour walk");
        // the first seven status words: the walk's own and the pass guard of
        // the bottom-up mass pass that ran before it
        static_assert(offsetof(DevStatus, pass_guard) == 6 * sizeof(int), "status word layout");
        SPHGPU_CUDA(c, cudaMemcpyAsync(&c->h_status, c->d_status, 7 * sizeof(int), cudaMemcpyDeviceToHost, st));
        SPHGPU_CUDA(c, cudaStreamSynchronize(st));
        if(c->h_status.fatal) {
            return fail(c, SPHGPU_ERR_NEIGHBOR_OVERFLOW,
                        "Neighbor list overflow: more than neighborNumber * 1000 neighbours");
        }
        {
            const int rcg = check_pass_guard(c);
            if(rcg < 0) return rcg;
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
    c->skin_valid = false;  // the exact lists replace any skin lists
    stage_begin(c, SPHGPU_T_GATHER_WALK);
    int launches = 0;
    const int rc = run_walk(c, 0, compute_guess, ratio, false, 0, &launches);
    stage_end(c, SPHGPU_T_GATHER_WALK, launches);
    return rc;
}

// ---------------------------------------------------------------------------
// Skin lists.  The step's true gather list of particle i is
//   { j : r_ij < R_i, box tests on the path }, R_i = ratio * the h guess,
// and every such j satisfies r_ij < R_i - delta or lies in the band replayed
// by box tests.  A list built with radius F_i >= R_i at positions x^b holds
// every j with |x_i^b - x_j^b| < F_i - delta.  Since
//   |x_i^b - x_j^b| <= r_ij + d_i + d_j  (d = displacement since the build,
//   minimum image),
// it holds the step's true list when R_i + d_i + d_max < F_i - delta for
// every i (d_max = the largest displacement).  Consumers take from a skin list
// exactly the members of the true list: pairs with r < h for h < R - delta
// need no other test (they are members); PreInteraction tests membership
// exactly for a particle whose h reaches R - delta, and the force-list build
// falls back to the symmetric walk for it.

namespace {

// The h guess into sml (the walk's expression, bit for bit), and the largest
// displacement since the build (rounded up).
__global__ void k_skin_guess(DevParams P, DevState S, int n, double ratio, const double4* __restrict__ xb,
                             double* __restrict__ dmax)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double d = 0.0;
    if(i < n) {
        const double4 p = S.pos[i];
        constexpr double A = 4.0 * 3.14159265358979323846 / 3.0;
        S.vel[i].w = pow(P.nngb * p.w / (S.thermo[i].x * A), 1.0 / 3) * ratio;
        const double4 b = xb[i];
        const Vec3d v = rij(P, p.x, p.y, p.z, b.x, b.y, b.z);
        d = sqrt(v.x * v.x + v.y * v.y + v.z * v.z) * (1.0 + 1e-12);
    }
    d = warp_max_pos(d);
    if((threadIdx.x & 31) == 0 && d > 0.0) atomic_max_pos(dmax, d);
}

__device__ __forceinline__ double skin_need_radius(const DevParams& P, const DevState& S, int i,
                                                   const double4* __restrict__ xb, double dmax, double delta)
{
    const double4 p = S.pos[i];
    const double4 b = xb[i];
    const Vec3d v = rij(P, p.x, p.y, p.z, b.x, b.y, b.z);
    const double d = sqrt(v.x * v.x + v.y * v.y + v.z * v.z) * (1.0 + 1e-12);
    return (S.vel[i].w + d + dmax) * (1.0 + 1e-12) + 2.0 * delta;
}

__global__ void k_skin_check(DevParams P, DevState S, int n, const double* __restrict__ fr,
                             const double4* __restrict__ xb, const double* __restrict__ dmax, double delta,
                             int* __restrict__ bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    if(!(skin_need_radius(P, S, i, xb, *dmax, delta) < fr[i])) *bad = 1;
}

// After a failed check: the largest skin any particle needed, in units of the
// gather radius the lists were built for (fr / factor), i.e. the largest
// need * factor / fr - 1 (one atomic per block of SKB).
constexpr int SKB = 256;
__global__ void __launch_bounds__(SKB) k_skin_need(DevParams P, DevState S, int n, const double* __restrict__ fr,
                                                   const double4* __restrict__ xb, const double* __restrict__ dmax,
                                                   double delta, double factor,
                                                   unsigned long long* __restrict__ need_max)
{
    __shared__ double sm[SKB / 32];
    const int i = blockIdx.x * SKB + threadIdx.x;
    double q = 0.0;
    if(i < n) {
        q = skin_need_radius(P, S, i, xb, *dmax, delta) * factor / fr[i] - 1.0;
        if(!(q >= 0.0)) q = 0.0;
    }
    q = warp_max_pos(q);
    if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = q;
    __syncthreads();
    if(threadIdx.x == 0) {
        for(int w = 1; w < SKB / 32; ++w) q = fmax(q, sm[w]);
        if(q > 0.0) atomicMax(need_max, (unsigned long long)__double_as_longlong(q));
    }
}

// Lists, counts, radii and build positions of the previous particle order
// moved to the order of the new tree (particle q now at p = new_of_old[q]).
__global__ void k_skin_compose(const uint32_t* __restrict__ src, const uint32_t* __restrict__ map, int n,
                               uint32_t* __restrict__ out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p < n) out[p] = map[src[p]];
}

__global__ void k_skin_new_of_old(const uint32_t* __restrict__ src, int n, int* __restrict__ new_of_old)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p < n) new_of_old[src[p]] = p;
}

__global__ void k_skin_permute(const uint32_t* __restrict__ src, int n, int cap, const int* __restrict__ new_of_old,
                               const int* __restrict__ list, const int* __restrict__ count, const double* __restrict__ fr,
                               const double4* __restrict__ xb, int* __restrict__ list2, int* __restrict__ count2,
                               double* __restrict__ fr2, double4* __restrict__ xb2)
{
    // one half-warp per row (8.78 M sphere: 4.3 -> 3.4 ms against a warp)
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const int lane = threadIdx.x & 15;
    if(w >= n) return;
    const int p = (int)w;
    const int q = (int)src[p];
    const int cnt = min(count[q], cap);
    const int* a = list + (size_t)q * (size_t)cap;
    int* b = list2 + (size_t)p * (size_t)cap;
    if((cap & 3) == 0) {
        // rows start on 16 bytes: up to four 16-byte loads of four entries
        // per lane, then their gathers, all in flight together (entries past
        // cnt are copied as is)
        const int4* a4 = reinterpret_cast<const int4*>(a);
        int4* b4 = reinterpret_cast<int4*>(b);
        for(int e0 = lane; 4 * e0 < cnt; e0 += 64) {
            int4 v[4];
            bool in[4];
#pragma unroll
            for(int t = 0; t < 4; ++t) {
                const int e = e0 + 16 * t;
                in[t] = 4 * e < cnt;
                v[t] = in[t] ? __ldg(&a4[e]) : make_int4(0, 0, 0, 0);
            }
#pragma unroll
            for(int t = 0; t < 4; ++t) {
                const int k = 4 * (e0 + 16 * t);
                if(!in[t]) continue;
                v[t].x = __ldg(&new_of_old[v[t].x]);
                if(k + 1 < cnt) v[t].y = __ldg(&new_of_old[v[t].y]);
                if(k + 2 < cnt) v[t].z = __ldg(&new_of_old[v[t].z]);
                if(k + 3 < cnt) v[t].w = __ldg(&new_of_old[v[t].w]);
            }
#pragma unroll
            for(int t = 0; t < 4; ++t)
                if(in[t]) b4[e0 + 16 * t] = v[t];
        }
    } else {
        for(int e = lane; e < cnt; e += 16) b[e] = __ldg(&new_of_old[__ldg(&a[e])]);
    }
    if(lane == 0) {
        count2[p] = cnt;
        fr2[p] = fr[q];
        xb2[p] = xb[q];
    }
}

}  // namespace

// The walk's safety margin (1e-12 of the domain scale) for the current tree,
// from its root box; 1e300 (no reuse) if it cannot be read.
double skin_delta(sphgpu_ctx* c)
{
    double4 root;
    if(cudaMemcpyAsync(&root, c->t.geo, sizeof(double4), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
       cudaStreamSynchronize(c->stream) != cudaSuccess)
        return 1e300;
    return 1e-12 * (std::max(std::fabs(root.x), std::max(std::fabs(root.y), std::fabs(root.z))) + root.w);
}

// Returns SPHGPU_OK, a CUDA failure (< 0), or 1 when the device has no room
// for the skin buffers (the caller then walks exactly instead).
int skin_alloc(sphgpu_ctx* c)
{
    // per-particle arrays (build radius and position, counts, permutation
    // scratch) follow n; the second list buffer follows n x capacity, and is
    // an allocation of its own: it trades places with d_glist at every
    // permutation
    const size_t n = (size_t)c->n;
    auto room = [&](void** p, size_t bytes) {
        if(cudaMalloc(p, bytes) == cudaSuccess) return true;
        (void)cudaGetLastError();  // an allocation failure is not sticky: clear it
        *p = nullptr;
        return false;
    };
    if(c->skin_n != c->n || !c->d_skin) {
        if(c->d_skin) {
            SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
            SPHGPU_CUDA(c, cudaFree(c->d_skin));
            c->d_skin = nullptr;
        }
        auto al = [](size_t b) { return (b + 255) / 256 * 256; };
        const size_t bytes = al(4 * n) + 2 * al(8 * n) + 2 * al(32 * n) + 3 * al(4 * n) + 256;
        c->skin_n = 0;
        if(!room(&c->d_skin, bytes)) return 1;
        char* b = static_cast<char*>(c->d_skin);
        size_t off = 0;
        auto take = [&](size_t sz) {
            char* q = b + off;
            off += al(sz);
            return q;
        };
        c->d_gcount_alt = reinterpret_cast<int*>(take(4 * n));
        c->d_skin_r = reinterpret_cast<double*>(take(8 * n));
        c->d_skin_r_alt = reinterpret_cast<double*>(take(8 * n));
        c->d_skin_x = reinterpret_cast<double4*>(take(32 * n));
        c->d_skin_x_alt = reinterpret_cast<double4*>(take(32 * n));
        c->d_skin_new = reinterpret_cast<int*>(take(4 * n));
        c->d_skin_map = reinterpret_cast<uint32_t*>(take(4 * n));
        c->d_skin_src = reinterpret_cast<uint32_t*>(take(4 * n));
        c->d_skin_scal = reinterpret_cast<double*>(take(24));
        c->skin_n = c->n;
        c->skin_valid = false;
        c->skin_map_pending = false;
    }
    if(c->skin_cap != c->gcap || !c->d_glist_alt) {
        if(c->d_glist_alt) {
            SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
            SPHGPU_CUDA(c, cudaFree(c->d_glist_alt));
            c->d_glist_alt = nullptr;
        }
        c->skin_cap = 0;
        if(!room(reinterpret_cast<void**>(&c->d_glist_alt), std::max<size_t>(4 * n * (size_t)c->gcap, 4))) return 1;
        c->skin_cap = c->gcap;
    }
    return SPHGPU_OK;
}

int skin_permute(sphgpu_ctx* c, const uint32_t* src)
{
    if(!c->skin_valid) return SPHGPU_OK;
    if(c->skin_n != c->n || c->skin_cap != c->gcap) {
        c->skin_valid = false;
        return SPHGPU_OK;
    }
    const int n = c->n;
    if(c->skin_map_pending) {
        // an upload put the particles in caller order since the lists were
        // last moved: compose that step with this one
        k_skin_compose<<<grid_for(n, 256), 256, 0, c->stream>>>(src, c->d_skin_map, n, c->d_skin_src);
        src = c->d_skin_src;
        c->skin_map_pending = false;
    }
    k_skin_new_of_old<<<grid_for(n, 256), 256, 0, c->stream>>>(src, n, c->d_skin_new);
    k_skin_permute<<<grid_for((long long)n * 16, 256), 256, 0, c->stream>>>(
        src, n, (int)c->gcap, c->d_skin_new, c->d_glist, c->d_gcount, c->d_skin_r, c->d_skin_x, c->d_glist_alt,
        c->d_gcount_alt, c->d_skin_r_alt, c->d_skin_x_alt);
    SPHGPU_LAUNCH_CHECK(c, "skin list permutation");
    std::swap(c->d_glist, c->d_glist_alt);
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_gcount, c->d_gcount_alt, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice,
                                   c->stream));
    std::swap(c->d_skin_r, c->d_skin_r_alt);
    std::swap(c->d_skin_x, c->d_skin_x_alt);
    c->stage_launch[SPHGPU_T_TREE] += 2;
    c->launches += 2;
    return SPHGPU_OK;
}

int skin_upload(sphgpu_ctx* c)
{
    // the lists keep their rows; the row of the particle now at caller index
    // k is its octree position before the upload (inv), applied at the next
    // tree build together with that build's own permutation
    if(!c->skin_valid || c->skin_map_pending) return SPHGPU_OK;
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_skin_map, c->d_inv, sizeof(int) * (size_t)c->n, cudaMemcpyDeviceToDevice,
                                   c->stream));
    c->skin_map_pending = true;
    return SPHGPU_OK;
}

int gather_lists(sphgpu_ctx* c, double ratio)
{
    constexpr int SKIN_PAUSE = 32;     // steps of exact walks after two unused builds
    constexpr double SKIN_GROW = 5.0;  // the widest skin, in units of gather_skin
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "neighbour search before tree make");
    const double skin = c->prm.gather_skin;
    if(!(skin > 0.0) || c->walk_mode != 0) return gather_walk(c, true, ratio);
    if(c->skin_off > 0) {
        // lists that were not reused twice in a row: exact walks for a while
        --c->skin_off;
        return gather_walk(c, true, ratio);
    }
    cudaStream_t st = c->stream;
    const int n = c->n;
    c->skin_delta_now = skin_delta(c);
    if(!(c->skin_delta_now < 1e299)) return gather_walk(c, true, ratio);
    if(c->skin_valid) {
        stage_begin(c, SPHGPU_T_GATHER_WALK);
        // {largest displacement, failed-check flag, largest skin needed}
        double* dmax = c->d_skin_scal;
        int* bad = reinterpret_cast<int*>(c->d_skin_scal + 1);
        auto* need = reinterpret_cast<unsigned long long*>(c->d_skin_scal + 2);
        SPHGPU_CUDA(c, cudaMemsetAsync(c->d_skin_scal, 0, 24, st));
        k_skin_guess<<<grid_for(n, 256), 256, 0, st>>>(c->dp, c->s, n, ratio, c->d_skin_x, dmax);
        k_skin_check<<<grid_for(n, 256), 256, 0, st>>>(c->dp, c->s, n, c->d_skin_r, c->d_skin_x, dmax,
                                                        c->skin_delta_now, bad);
        SPHGPU_LAUNCH_CHECK(c, "skin check");
        int hbad = 1;
        SPHGPU_CUDA(c, cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPHGPU_CUDA(c, cudaStreamSynchronize(st));
        if(hbad) {
            k_skin_need<<<grid_for(n, SKB), SKB, 0, st>>>(c->dp, c->s, n, c->d_skin_r, c->d_skin_x, dmax,
                                                          c->skin_delta_now, c->skin_factor, need);
            SPHGPU_LAUNCH_CHECK(c, "skin need");
            double hneed = -1.0;
            SPHGPU_CUDA(c, cudaMemcpyAsync(&hneed, need, sizeof hneed, cudaMemcpyDeviceToHost, st));
            SPHGPU_CUDA(c, cudaStreamSynchronize(st));
            c->skin_need = hneed;
        }
        stage_end(c, SPHGPU_T_GATHER_WALK, hbad ? 3 : 2);
        if(!hbad) {
            ++c->skin_reuses;
            ++c->skin_since_build;
            return SPHGPU_OK;
        }
    }
    // two builds in a row whose lists served fewer than two steps: the next
    // build takes twice the skin (up to SKIN_GROW times gather_skin), when
    // the failed check shows that a skin within that bound would have served
    // two steps of the same motion; lists that served eight or more: half
    // (down to gather_skin).  A build whose lists were never reused and that
    // does not widen the skin was wasted work (the wider walk, the longer
    // lists); after two in a row the skin pauses
    if(c->skin_built) {
        const int used = c->skin_since_build;
        c->skin_short = used < 2 ? c->skin_short + 1 : 0;
        const double want = c->skin_need >= 0.0 ? 2.0 * c->skin_need / (double)(used + 1) / skin : 1e300;
        bool grow = c->skin_short >= 2 && c->skin_scale < SKIN_GROW && want <= SKIN_GROW;
        if(grow) {
            // wider lists need longer rows in both list buffers: widen only
            // with twice the present buffers free (a second buffer that no
            // longer fits would end the skin lists for good)
            size_t free_b = 0, total_b = 0;
            const size_t lists_b = 2 * sizeof(int) * (size_t)n * (size_t)c->gcap;
            if(cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < 2 * lists_b) grow = false;
        }
        if(grow)
            c->skin_scale = std::min(2.0 * c->skin_scale, SKIN_GROW);
        else if(used >= 8)
            c->skin_scale = std::max(0.5 * c->skin_scale, 1.0);
        c->skin_idle = !grow && used == 0 ? c->skin_idle + 1 : 0;
    } else {
        c->skin_idle = 0;
    }
    c->skin_since_build = 0;
    c->skin_need = -1.0;
    if(c->skin_idle >= 2) {
        c->skin_idle = 0;
        c->skin_off = SKIN_PAUSE - 1;
        return gather_walk(c, true, ratio);
    }
    // build: the walk at radius (1 + skin) R, recording radii and positions
    int rc = ensure_list_capacity(c, 0, c->gcap);
    if(rc < 0) return rc;
    rc = skin_alloc(c);
    if(rc < 0) return rc;
    if(rc == 1) {
        // no room for a second list buffer: exact walks from here on
        c->skin_valid = false;
        c->skin_off = 1 << 30;
        return gather_walk(c, true, ratio);
    }
    c->skin_valid = false;
    stage_begin(c, SPHGPU_T_GATHER_WALK);
    int launches = 0;
    c->skin_factor = 1.0 + skin * c->skin_scale;
    rc = run_walk(c, 0, true, ratio, false, 0, &launches, SkinOut{c->skin_factor, c->d_skin_r, c->d_skin_x});
    stage_end(c, SPHGPU_T_GATHER_WALK, launches);
    if(rc == SPHGPU_ERR_NEIGHBOR_OVERFLOW) return gather_walk(c, true, ratio);  // decided on the exact lists
    if(rc < 0) return rc;
    // the walk may have grown the list capacity: the second list buffer
    // follows (the recorded radii and positions are per particle and stand)
    const int ra = skin_alloc(c);
    if(ra < 0) return ra;
    if(ra == 1) {
        // the grown lists leave no room for their second buffer: these lists
        // are skin lists (supersets) and must not be taken as exact ones
        c->skin_off = 1 << 30;
        return gather_walk(c, true, ratio);
    }
    c->skin_valid = true;
    c->skin_built = true;
    ++c->skin_builds;
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
    DevTemps tmp(st);
    SPHGPU_CUDA(c, tmp.get(&d_cnt, sizeof(unsigned long long) * (size_t)(2 * n + 2)));
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
            SPHGPU_CUDA(c, tmp.get(&d_ids, sizeof(int) * (size_t)(total + 1)));
            k_fill_by_id<<<grid_for(n, 256), 256, 0, st>>>(n, (int)lcap, c->s.id, count, list, d_off, d_ids);
            SPHGPU_CUDA(c, cudaMemcpyAsync(ids, d_ids, sizeof(int) * (size_t)total, cudaMemcpyDeviceToHost, st));
        }
    }
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
