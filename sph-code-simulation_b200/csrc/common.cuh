// common.cuh — device-side building blocks shared by every kernel file.
//
// Data layout in HBM (all arrays in octree / Morton order, length n).
// Fields are packed four to a double4 by the stage that reads them together,
// so a neighbour's inputs to a pair loop arrive in 32-byte sectors:
//   pos    {x, y, z, mass}
//   vel    {vx, vy, vz, sml}
//   acc    {ax, ay, az, dene}
//   velp   {vpx, vpy, vpz, ene_p}        (predictor half step)
//   thermo {dens, pres, ene, sound}
//   visc   {alpha, balsara, gradh, phi}
//   grad   4 x n double4: GSPH MUSCL gradients of rho (3), P (3), v_x (3),
//          v_y (3), v_z (3) packed in that order (15 used slots)
//   id     int32  caller index of the particle (the reference's vector index)
//   nbr    int32  neighbour count of the last PreInteraction
//   sr     srgsph only, 4 x n double4: {S, e}, {N, nu, gamma_lor, enthalpy},
//          {dS/dt, de/dt}, {N before the current pre-interaction}
// Octree nodes are stored in depth-first preorder (children in index order
// 0..7, the order of BHNode::childs, include/bhtree.hpp:19-31) so a walk is a
// forward scan with `skip` pointers over whole subtrees.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sphgpu.h"

namespace sphgpu {

constexpr unsigned FULL_MASK = 0xffffffffu;

// ------------------------------------------------------------ parameters
struct DevParams {
    int sph_type, kernel, nngb, iterative;
    double gamma, cfl_sound, cfl_force, av_alpha;
    int balsara, td_av;
    double alpha_max, alpha_min, eps_av;
    int use_ac;
    double alpha_ac;
    int max_level, leaf_num;
    int periodic;
    int root_origin;  // non-periodic root box also covers the origin
    double lo[3], hi[3], range[3];
    int gravity;
    double G, theta, theta2;
    int gsph2, riemann, precision, guess, mlp_max_newton;
    double ratio;  // kernel ratio 1.2 (iterative sml) or 1.0 (src/pre_interaction.cpp:31-35)
    int sr_2nd;    // srgsph: MUSCL reconstruction
    double sr_c, sr_c_shock, sr_c_cd, sr_eta, sr_c_smooth;
    double mixed_acc_tol;  // mixed form: FP64 re-evaluation above this estimated error
    double riemann_tol;    // plain iterative Riemann solver: stop at this relative change of p
    double gather_skin;    // skin of the reused gather lists (0 = exact walk every step)
};

struct DevState {
    int n;
    double4* pos;
    double4* vel;
    double4* acc;
    double4* velp;
    double4* thermo;
    double4* visc;
    double4* grad;  // 4 * n
    int* id;
    int* nbr;
    // srgsph only (null otherwise), 4 * n: {S x, y, z, e}, {N, nu, gamma_lor,
    // enthalpy}, {dS/dt x, y, z, de/dt}, {N before the current pre-interaction, -, -, -}
    double4* sr;
};

struct DevTree {
    double4* geo;    // center x, y, z, edge
    double4* mass;   // centre of mass x, y, z, mass
    double* ksize;   // kernel_size: max sml in the subtree
    int4* link;      // start, end, skip, level | is_leaf << 8
    int* child;      // 8 slots per node (child index by octant, -1 = none)
    int* parent;
    int* nchild;
    int* counter;
    int* nnodes;     // device scalar: total node count (root included)
    int* leaf_of;    // per particle (tree order): the leaf holding it
    double* pks;     // per particle: kernel_size of its leaf (set_kernel)
};

// Packed status words read back by the host after a module.
struct DevStatus {
    int overflow;          // a neighbour list exceeded the current capacity
    int fatal;             // a list exceeded neighbor_number * 1000
    int max_count;         // largest list seen
    int node_pool;         // node pool exhausted
    int guard;             // a neighbour walk hit its node-count bound (corrupt tree)
    int nonfinite;         // a particle position is NaN or infinite
    int pass_guard;        // PASS_GUARD_* bits: a bottom-up pass or gravity walk hit its bound
    unsigned long long newton_nonconv;
    unsigned long long riemann_solves;
    unsigned long long riemann_iters;
    unsigned long long riemann_fallbacks;
    unsigned long long walk_group_warps;   // warps that took the group walk
    unsigned long long walk_split_warps;   // warps walked as several sub-groups
    unsigned long long mlp_guesses;        // pairs sent to the learned guess
    int sr_recovery;                       // srgsph: a Lorentz-factor solve did not converge
    // work counters (units of the FLOP roofline; reset with the others)
    unsigned long long pre_cand;           // gather-list candidates tested (every sweep + fused pass)
    unsigned long long pre_newton_pairs;   // pairs inside h in the Newton sweeps
    unsigned long long pre_pairs;          // pairs inside h in the fused pass
    unsigned long long pre_list;           // gather-list entries (each list read once: the fused pass)
    unsigned long long force_cand;         // pair-list entries tested by FluidForce
    unsigned long long force_pairs;        // pairs inside max(h_i, h_j)
    unsigned long long grav_nodes;         // nodes met by the gravity walk (opening tests)
    unsigned long long grav_mono;          // nodes accepted as monopoles
    unsigned long long grav_leaf_pairs;    // softened particle pairs in opened leaves
};

// Sum a per-lane work counter over the block and add it to a device total
// (one atomic per block).  Every thread of the block must call it.
__device__ __forceinline__ void block_count(unsigned long long* total, unsigned v)
{
    __shared__ unsigned long long s_cnt[32];
    unsigned long long x = v;
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if((threadIdx.x & 31) == 0) s_cnt[w] = x;
    __syncthreads();
    if(threadIdx.x == 0) {
        unsigned long long t = 0;
        for(int k = 0; k < (int)((blockDim.x + 31) >> 5); ++k) t += s_cnt[k];
        if(t) atomicAdd(total, t);
    }
}

// Bits of DevStatus::pass_guard.  The passes that set them run without a
// host wait after them; the host reports the bit at its next wait on the
// stream (check_pass_guard in capi.cu).
constexpr int PASS_GUARD_MASS = 1;       // bottom-up mass / centre of mass
constexpr int PASS_GUARD_KSIZE = 2;      // bottom-up kernel_size (set_kernel)
constexpr int PASS_GUARD_GRAVITY = 4;    // Barnes-Hut walk (FP64)
constexpr int PASS_GUARD_GRAVITY32 = 8;  // Barnes-Hut walk (mixed form)

// Read-only 32-byte load through the non-coherent path, one 256-bit access
// (sm_100).  p must be 32-byte aligned: every double4 array here is an
// allocation of its own (256-byte aligned) indexed by element.  Only for data
// that no thread of the kernel writes (the non-coherent path may return an
// older value of a location written during the kernel).
__device__ __forceinline__ double4 ldg4(const double4* p)
{
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

// ------------------------------------------------------------ exact FP64
// The reference is compiled for x86-64 without FMA contraction; expressions
// that decide set membership or tree topology use explicitly rounded
// operations so they evaluate exactly as there.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }

// Periodic::calc_r_ij (include/periodic.hpp:34-59), one axis: candidates
// d, d + L, d - L with the first minimal |.| winning ties.  Fast path: for
// |d| <= L/2 the reference always keeps d (|d + L| and |d - L| are then
// >= L/2 >= |d|, and a tie keeps the first candidate), so the other two
// candidates need not be formed.
__device__ __forceinline__ double min_image(double d, double L)
{
    if(fabs(d) <= 0.5 * L) return d;
    const double b = xadd(d, L), c = xsub(d, L);
    const double ad = fabs(d), ab = fabs(b), ac = fabs(c);
    if(ad <= ab && ad <= ac) return d;
    if(ab <= ac && ab <= ad) return b;
    if(ac <= ad && ac <= ab) return c;
    return d;
}

struct Vec3d {
    double x, y, z;
};

__device__ __forceinline__ Vec3d rij(const DevParams& P, double xi, double yi, double zi,
                                     double xj, double yj, double zj)
{
    Vec3d d{xsub(xi, xj), xsub(yi, yj), xsub(zi, zj)};
    if(P.periodic) {
        d.x = min_image(d.x, P.range[0]);
        d.y = min_image(d.y, P.range[1]);
        d.z = min_image(d.z, P.range[2]);
    }
    return d;
}

// abs2 (include/vector_type.hpp:227-230): ((x*x + y*y) + z*z), unfused.
__device__ __forceinline__ double abs2x(Vec3d d)
{
    return xadd(xadd(xmul(d.x, d.x), xmul(d.y, d.y)), xmul(d.z, d.z));
}

// Membership of j in the reference's gather list of i (radius R), for a
// particle whose h reaches R - delta while its candidates come from a skin
// list (a superset): r^2 < R^2 and, within delta of the radius, the
// reference's box tests up the path from j's leaf (src/bhtree.cpp:277-316), in
// unfused FP64 as the walk evaluates them.  Rare.
__device__ __forceinline__ bool gather_member_x(const double4* __restrict__ geo, const int* __restrict__ parent,
                                             const int* __restrict__ leaf_of, int periodic, double Lx, double Ly,
                                             double Lz, double xi, double yi, double zi, double R, double delta, int j,
                                             double r2)
{
    if(!(r2 < xmul(R, R))) return false;
    const double hs = R - delta;
    if(hs > 0.0 && r2 < xmul(hs, hs)) return true;
    int A = __ldg(&leaf_of[j]);
    for(int up = 0; A >= 0 && up < 64; ++up) {
        const double4 g = ldg4(&geo[A]);
        const double e = xadd(xmul(g.w, 0.5), R);
        double dx = xsub(xi, g.x), dy = xsub(yi, g.y), dz = xsub(zi, g.z);
        if(periodic) {
            dx = min_image(dx, Lx);
            dy = min_image(dy, Ly);
            dz = min_image(dz, Lz);
        }
        const double m = fmax(fmax(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
        if(!(m <= xmul(e, e))) return false;
        A = A == 0 ? -1 : __ldg(&parent[A]);
    }
    return true;
}

__device__ __forceinline__ bool gather_member(const DevParams& P, const DevTree& T, double xi, double yi, double zi,
                                              double R, double delta, int j, double r2)
{
    return gather_member_x(T.geo, T.parent, T.leaf_of, P.periodic, P.range[0], P.range[1], P.range[2], xi, yi, zi,
                           R, delta, j, r2);
}

// The reference's pair predicate r < h with r = sqrt(r^2) correctly rounded
// (src/pre_interaction.cpp:89, src/fluid_force.cpp:62), decided from r^2:
// outside a band of relative width 2^-40 around h^2 the rounding of the root
// cannot change the answer (2^-40 is far above the 2^-53 rounding of h * h and
// of the root), so the square root is taken only inside the band.
__device__ __forceinline__ bool root_lt(double r2, double h)
{
    const double h2 = h * h;
    if(r2 < h2 * (1.0 - 0x1p-40)) return true;
    if(r2 > h2 * (1.0 + 0x1p-40)) return false;
    return sqrt(r2) < h;
}

// Pair loops: true when sqrt(r2) < h (exactly as root_lt); then r and 1/r.
// Outside the band they come from one reciprocal square root (CUDA's rsqrt,
// within an ulp of 1/sqrt), inside it from the correctly rounded root; for
// r2 = 0 both are 0.  The pair sums built from them agree with the
// reference's to rounding, as before; only set membership must be exact.
__device__ __forceinline__ bool pair_within(double r2, double h, double& r, double& rinv)
{
    const double h2 = h * h;
    if(r2 > h2 * (1.0 + 0x1p-40)) return false;
    if(r2 >= h2 * (1.0 - 0x1p-40)) {
        r = sqrt(r2);
        if(!(r < h)) return false;
        rinv = r > 0.0 ? 1.0 / r : 0.0;
        return true;
    }
    if(r2 > 0.0) {
        rinv = rsqrt(r2);
        r = r2 * rinv;
    } else {
        r = 0.0;
        rinv = 0.0;
    }
    return true;
}

// ------------------------------------------------------------ SPH kernels
// W, grad W (as the scalar c with grad W = r_ij c) and dW/dh for the cubic
// spline (include/kernel/cubic_spline.hpp:21-53), Wendland C4
// (include/kernel/wendland_kernel.hpp:23-49) and the Gaussian
// W = exp(-(r/h)^2) / (h^3 pi^(3/2)) that the reference cuts at r = h like the
// others (include/kernel/gaussian_kernel.hpp:21-57), DIM = 3, restated from the
// formulas; T = double (plain form) or float (mixed form).
// 1 / pi^(3/2) as the reference writes it (to 15 digits)
constexpr double GAUSS_SIGMA = 0.179587122125167;
template <typename T>
struct Kern {
    static constexpr double PI = 3.14159265358979323846;
    __device__ static __forceinline__ T cube(T x) { return x * x * x; }
    __device__ static __forceinline__ T pow5(T x) { return x * x * x * x * x; }
    __device__ static __forceinline__ T pow6(T x) { return x * x * x * x * x * x; }

    __device__ static __forceinline__ T w(int type, T r, T h)
    {
        if(type == SPHGPU_GAUSSIAN) {
            const T q = r / h;
            return T(GAUSS_SIGMA) / cube(h) * exp(-(q * q));
        }
        if(type == SPHGPU_WENDLAND) {
            const T sigma = T(495.0 / (32.0 * PI));
            const T q = r / h;
            const T a = T(0.5) * (T(1) - q + fabs(T(1) - q));
            return sigma / cube(h) * pow6(a) * (T(1) + T(6) * q + T(35.0 / 3.0) * q * q);
        }
        const T sigma = T(1.0 / PI);
        const T hh = h * T(0.5);
        const T q = r / hh;
        const T a = T(0.5) * (T(2) - q + fabs(T(2) - q));
        const T b = T(0.5) * (T(1) - q + fabs(T(1) - q));
        return sigma / cube(hh) * (T(0.25) * cube(a) - cube(b));
    }

    __device__ static __forceinline__ T dwc(int type, T r, T h)
    {
        if(type == SPHGPU_GAUSSIAN) {
            if(r == T(0)) return T(0);
            const T q = r / h;
            const T wv = T(GAUSS_SIGMA) / cube(h) * exp(-(q * q));
            return T(-2) * wv * q / (h * r);
        }
        if(type == SPHGPU_WENDLAND) {
            const T sigma = T(495.0 / (32.0 * PI));
            const T q = r / h;
            const T a = T(0.5) * (T(1) - q + fabs(T(1) - q));
            return T(-56.0 / 3.0) * sigma / (cube(h) * (h * h)) * pow5(a) * (T(1) + T(5) * q);
        }
        if(r == T(0)) return T(0);
        const T sigma = T(1.0 / PI);
        const T hh = h * T(0.5);
        const T q = r / hh;
        const T a = T(0.5) * (T(2) - q + fabs(T(2) - q));
        const T b = T(0.5) * (T(1) - q + fabs(T(1) - q));
        return -sigma / (cube(hh) * hh * r) * (T(0.75) * (a * a) - T(3) * (b * b));
    }

    __device__ static __forceinline__ T dhw(int type, T r, T h)
    {
        if(type == SPHGPU_GAUSSIAN) {
            const T q = r / h;
            const T wv = T(GAUSS_SIGMA) / cube(h) * exp(-(q * q));
            return wv * (T(2) * (q * q) - T(3)) / h;
        }
        if(type == SPHGPU_WENDLAND) {
            const T sigma = T(495.0 / (32.0 * PI));
            const T q = r / h;
            const T a = T(0.5) * (T(1) - q + fabs(T(1) - q));
            return -sigma / (cube(h) * h * T(3)) * pow5(a)
                * (T(9) + T(45) * q + T(-5) * q * q - T(385) * cube(q));
        }
        const T sigma = T(1.0 / PI);
        const T hh = h * T(0.5);
        const T q = r / hh;
        const T a = T(0.5) * (fabs(T(2) - q) + T(2) - q);
        const T b = T(0.5) * (fabs(T(1) - q) + T(1) - q);
        return T(0.5) * sigma / (cube(hh) * hh) * (a * a * (T(1.5) * q - T(1.5)) + b * b * (T(-6) * q + T(3)));
    }
};

// The same kernels with the h-dependent factors hoisted out of the pair loop
// (one set per smoothing length): the pair then costs multiplications only,
// plus 1/r for the cubic gradient.  Results differ from Kern<T> by rounding.
template <typename T>
struct KernH {
    T inv;   // 1/h (Wendland) or 1/(h/2) (cubic)
    T wn;    // W = wn * shape(q)
    T dwn;   // grad W = r_ij * dwn * shape'(q)  (cubic: times 1/r)
    T dhn;   // dW/dh = dhn * shape_h(q)
    int type;

    __device__ __forceinline__ KernH(int type_, T h) : type(type_)
    {
        constexpr double PI = 3.14159265358979323846;
        if(type == SPHGPU_GAUSSIAN) {
            inv = T(1) / h;
            wn = T(GAUSS_SIGMA) * inv * inv * inv;
            dwn = T(-2) * wn * inv;  // times q / r
            dhn = wn * inv;
            return;
        }
        if(type == SPHGPU_WENDLAND) {
            const T sigma = T(495.0 / (32.0 * PI));
            inv = T(1) / h;
            const T i3 = inv * inv * inv;
            wn = sigma * i3;
            dwn = T(-56.0 / 3.0) * sigma * i3 * inv * inv;
            dhn = -sigma * i3 * inv * T(1.0 / 3.0);
        } else {
            const T sigma = T(1.0 / PI);
            inv = T(2) / h;
            const T i3 = inv * inv * inv;
            wn = sigma * i3;
            dwn = -sigma * i3 * inv;
            dhn = T(0.5) * sigma * i3 * inv;
        }
    }
    __device__ __forceinline__ T w(T r) const
    {
        const T q = r * inv;
        if(type == SPHGPU_GAUSSIAN) return wn * exp(-(q * q));
        if(type == SPHGPU_WENDLAND) {
            const T a = T(0.5) * (T(1) - q + fabs(T(1) - q));
            const T a2 = a * a;
            return wn * (a2 * a2 * a2) * (T(1) + T(6) * q + T(35.0 / 3.0) * q * q);
        }
        const T a = T(0.5) * (T(2) - q + fabs(T(2) - q));
        const T b = T(0.5) * (T(1) - q + fabs(T(1) - q));
        return wn * (T(0.25) * a * a * a - b * b * b);
    }
    __device__ __forceinline__ T dwc(T r, T rinv) const
    {
        const T q = r * inv;
        if(type == SPHGPU_GAUSSIAN) return r == T(0) ? T(0) : dwn * exp(-(q * q)) * q * rinv;
        if(type == SPHGPU_WENDLAND) {
            const T a = T(0.5) * (T(1) - q + fabs(T(1) - q));
            const T a2 = a * a;
            return dwn * (a2 * a2 * a) * (T(1) + T(5) * q);
        }
        if(r == T(0)) return T(0);
        const T a = T(0.5) * (T(2) - q + fabs(T(2) - q));
        const T b = T(0.5) * (T(1) - q + fabs(T(1) - q));
        return dwn * rinv * (T(0.75) * a * a - T(3) * b * b);
    }
    __device__ __forceinline__ T dhw(T r) const
    {
        const T q = r * inv;
        if(type == SPHGPU_GAUSSIAN) return dhn * exp(-(q * q)) * (T(2) * (q * q) - T(3));
        if(type == SPHGPU_WENDLAND) {
            const T a = T(0.5) * (T(1) - q + fabs(T(1) - q));
            const T a2 = a * a;
            return dhn * (a2 * a2 * a) * (T(9) + T(45) * q + T(-5) * q * q - T(385) * q * q * q);
        }
        const T a = T(0.5) * (T(2) - q + fabs(T(2) - q));
        const T b = T(0.5) * (T(1) - q + fabs(T(1) - q));
        return dhn * (a * a * (T(1.5) * q - T(1.5)) + b * b * (T(-6) * q + T(3)));
    }
};

// ------------------------------------------------------------ reductions
// Butterfly reductions over an aligned group of G lanes.  The shuffle mask
// names only the group's own lanes: groups of one warp may leave a loop at
// different iterations (per-particle Newton convergence), so a warp-wide
// mask would wait for lanes that never arrive.  All lanes of a group take
// identical control flow and end with the same bits.
template <int G>
__device__ __forceinline__ unsigned group_mask()
{
    if(G == 32) return FULL_MASK;
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
}
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v)
{
    const unsigned m = group_mask<G>();
#pragma unroll
    for(int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o, G);
    return v;
}
template <int G, typename T>
__device__ __forceinline__ T group_max(T v)
{
    const unsigned m = group_mask<G>();
#pragma unroll
    for(int o = G / 2; o > 0; o >>= 1) {
        const T u = __shfl_xor_sync(m, v, o, G);
        v = u > v ? u : v;
    }
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) {
        const T u = __shfl_xor_sync(FULL_MASK, v, o);
        v = u < v ? u : v;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max_pos(T v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) {
        const T u = __shfl_xor_sync(FULL_MASK, v, o);
        v = u > v ? u : v;
    }
    return v;
}

// Positive doubles order like their bit patterns.
__device__ __forceinline__ void atomic_min_pos(double* addr, double v)
{
    atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_pos(double* addr, double v)
{
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

inline unsigned grid_for(long long n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace sphgpu
