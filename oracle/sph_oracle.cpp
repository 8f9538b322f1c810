// sph_oracle.cpp — CPU restatement of the reference's per-step SPH hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker: tests/ compare
// the CUDA path against it, and bench.py's cpu_baseline leg may time it.  It is
// never linked into, called by, or shipped with the product library.
//
// Parity pinning: tests/test_oracle_golden.py checks this restatement against
// (1) golden vectors produced by the reference's own compiled modules
//     (oracle/_ref/libsphref.so, generated by tests/golden/make_golden.py), and
// (2) the reference's shipped Evrard t=0 snapshot values recorded in the same
//     fixtures (sample/evrard/results_new/00000.dat, energy.dat row t=0).
//
// Layout: structure-of-arrays (one std::vector<double> per particle field),
// particles addressed by index; the octree is an index-based node pool whose
// per-node particle lists are threaded through a `next` index array, because
// the order of those lists fixes the floating-point summation order of the
// node mass / centre of mass and of the gravity walk, and the order of the
// raw neighbour lists (src/bhtree.cpp:154-247).
//
// Arithmetic: every expression keeps the reference's operation order and is
// compiled with -ffp-contract=off, so results are bit-identical to the
// reference build on the same inputs wherever the reference is deterministic.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "sphgpu.h"

namespace oracle {

typedef double real;

inline real sqr(real x) { return x * x; }
inline real pow3(real x) { return x * x * x; }
inline real pow5(real x) { return x * x * x * x * x; }
inline real pow6(real x) { return x * x * x * x * x * x; }

struct V3 {
    real x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, real s) { return {a.x * s, a.y * s, a.z * s}; }
inline real dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline real norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline real comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// ---------------------------------------------------------------- kernels
// include/kernel/cubic_spline.hpp:21-53 (DIM = 3, sigma = 1/pi, support h).
struct CubicSpline {
    static constexpr real sigma = 1.0 / M_PI;
    static real w(real r, real h)
    {
        const real hh = h * 0.5;
        const real q = r / hh;
        const real a = 0.5 * (2.0 - q + std::abs(2.0 - q));
        const real b = 0.5 * (1.0 - q + std::abs(1.0 - q));
        return sigma / pow3(hh) * (0.25 * pow3(a) - pow3(b));
    }
    // returns the scalar c with grad W = r_ij * c
    static real dw(real r, real h)
    {
        if(r == 0.0) return 0.0;
        const real hh = h * 0.5;
        const real q = r / hh;
        const real a = 0.5 * (2.0 - q + std::abs(2.0 - q));
        const real b = 0.5 * (1.0 - q + std::abs(1.0 - q));
        return -sigma / (pow3(hh) * hh * r) * (0.75 * sqr(a) - 3.0 * sqr(b));
    }
    static real dhw(real r, real h)
    {
        const real hh = h * 0.5;
        const real q = r / hh;
        return 0.5 * sigma / (pow3(hh) * hh)
            * (sqr((std::abs(2.0 - q) + 2.0 - q) * 0.5) * ((3. + 3) * 0.25 * q - 0.5 * 3)
               + sqr((std::abs(1.0 - q) + 1.0 - q) * 0.5) * ((-3.0 - 3) * q + 3));
    }
};

// include/kernel/wendland_kernel.hpp:23-49 (Wendland C4, DIM = 3).
struct WendlandC4 {
    static constexpr real sigma = 495. / (32 * M_PI);
    static real w(real r, real h)
    {
        const real q = r / h;
        return sigma / pow3(h) * pow6(0.5 * (1.0 - q + std::abs(1.0 - q))) * (1.0 + 6.0 * q + 35.0 / 3.0 * q * q);
    }
    static real dw(real r, real h)
    {
        const real q = r / h;
        return -56.0 / 3.0 * sigma / (pow3(h) * sqr(h)) * pow5(0.5 * (1.0 - q + std::abs(1.0 - q))) * (1.0 + 5.0 * q);
    }
    static real dhw(real r, real h)
    {
        const real q = r / h;
        return -sigma / (pow3(h) * h * 3.0) * pow5(0.5 * (1.0 - q + std::abs(1.0 - q)))
            * (3.0 * 3 + 15.0 * 3 * q + (-56.0 + 17.0 * 3) * q * q - 35.0 * (8.0 + 3) * pow3(q));
    }
};

// include/kernel/gaussian_kernel.hpp:21-57 (DIM = 3): W = sigma / h^3 exp(-q^2),
// sigma = 1 / pi^(3/2) written to 15 digits as the reference writes it.
struct Gauss {
    static constexpr real sigma = 0.179587122125167;
    static real w(real r, real h)
    {
        const real q = r / h;
        const real q2 = q * q;
        return sigma / pow3(h) * std::exp(-q2);
    }
    static real dw(real r, real h)
    {
        if(r == 0.0) return 0.0;
        const real q = r / h;
        const real q2 = q * q;
        const real wv = sigma / pow3(h) * std::exp(-q2);
        return -2.0 * wv * q / (h * r);
    }
    static real dhw(real r, real h)
    {
        const real q = r / h;
        const real q2 = q * q;
        const real wv = sigma / pow3(h) * std::exp(-q2);
        return wv * (2.0 * q2 - static_cast<real>(3)) / h;
    }
};

struct Kernel {
    int type;
    real w(real r, real h) const
    {
        return type == SPHGPU_WENDLAND ? WendlandC4::w(r, h) : type == SPHGPU_GAUSSIAN ? Gauss::w(r, h) : CubicSpline::w(r, h);
    }
    real dwc(real r, real h) const
    {
        return type == SPHGPU_WENDLAND ? WendlandC4::dw(r, h) : type == SPHGPU_GAUSSIAN ? Gauss::dw(r, h) : CubicSpline::dw(r, h);
    }
    V3 dw(V3 rij, real r, real h) const { return rij * dwc(r, h); }
    real dhw(real r, real h) const
    {
        return type == SPHGPU_WENDLAND ? WendlandC4::dhw(r, h) : type == SPHGPU_GAUSSIAN ? Gauss::dhw(r, h) : CubicSpline::dhw(r, h);
    }
};

// ---------------------------------------------------------------- periodic
// include/periodic.hpp:34-72: one flag for all axes, three-candidate minimum
// image chosen in the order (r, r+L, r-L) with <= ties to the earlier one.
struct Periodic {
    bool valid = false;
    real lo[3], hi[3], range[3];
    real axis(real d, int k) const
    {
        const real a = d, b = d + range[k], c = d - range[k];
        if(std::abs(a) <= std::abs(b) && std::abs(a) <= std::abs(c)) return a;
        if(std::abs(b) <= std::abs(c) && std::abs(b) <= std::abs(a)) return b;
        if(std::abs(c) <= std::abs(a) && std::abs(c) <= std::abs(b)) return c;
        return a;  // NaN input: the reference asserts; keep the plain difference
    }
    V3 rij(V3 ri, V3 rj) const
    {
        V3 d = ri - rj;
        if(!valid) return d;
        return {axis(d.x, 0), axis(d.y, 1), axis(d.z, 2)};
    }
    void apply(real& x, int k) const
    {
        if(!valid) return;
        if(x < lo[k]) x += range[k];
        else if(x > hi[k]) x -= range[k];
    }
};

// ---------------------------------------------------------------- state
struct State {
    int n = 0;
    std::vector<real> f[SPHGPU_NFIELDS];
    std::vector<int> neighbor;
    real& at(int k, int i) { return f[k][i]; }
    V3 pos(int i) const { return {f[SPHGPU_F_POS_X][i], f[SPHGPU_F_POS_Y][i], f[SPHGPU_F_POS_Z][i]}; }
    V3 vel(int i) const { return {f[SPHGPU_F_VEL_X][i], f[SPHGPU_F_VEL_Y][i], f[SPHGPU_F_VEL_Z][i]}; }
    V3 acc(int i) const { return {f[SPHGPU_F_ACC_X][i], f[SPHGPU_F_ACC_Y][i], f[SPHGPU_F_ACC_Z][i]}; }
    V3 grad(int g, int i) const
    {
        const int b = SPHGPU_F_GRAD_D_X + 3 * g;
        return {f[b][i], f[b + 1][i], f[b + 2][i]};
    }
    void set_grad(int g, int i, V3 v)
    {
        const int b = SPHGPU_F_GRAD_D_X + 3 * g;
        f[b][i] = v.x;
        f[b + 1][i] = v.y;
        f[b + 2][i] = v.z;
    }
};

// ---------------------------------------------------------------- octree
// src/bhtree.cpp: the node pool, the particle lists threaded through `next`
// (assign prepends, so a node's list order alternates between ascending and
// descending particle index with depth), bottom-up mass and centre of mass.
struct Node {
    int first;         // head of this node's particle list (-1 = empty)
    real mass;
    int num;
    int child[8];
    real center[3];
    real mcenter[3];
    real edge;
    int level;
    real kernel_size;
    bool is_leaf;
    void clear()
    {
        first = -1;
        mass = 0.0;
        num = 0;
        std::fill(child, child + 8, -1);
        center[0] = center[1] = center[2] = 0.0;
        mcenter[0] = mcenter[1] = mcenter[2] = 0.0;
        edge = 0.0;
        level = 0;
        kernel_size = 0.0;
        is_leaf = false;
    }
};

struct Tree {
    int max_level = 20, leaf_num = 1;
    bool root_origin = true;  // non-periodic root box also covers the origin
    std::vector<Node> pool;   // pool[0] is the root
    int used = 0;
    std::vector<int> next;
    bool built = false;
    std::string err;

    // BHNode::assign (src/bhtree.cpp:206-247)
    bool assign(int node, int p, const State& s)
    {
        Node& nd = pool[node];
        const real pos[3] = {s.f[SPHGPU_F_POS_X][p], s.f[SPHGPU_F_POS_Y][p], s.f[SPHGPU_F_POS_Z][p]};
        int index = 0, mask = 1;
        for(int k = 0; k < 3; ++k) {
            if(pos[k] > nd.center[k]) index |= mask;
            mask <<= 1;
        }
        int c = nd.child[index];
        if(c < 0) {
            if((int)pool.size() - used < 0 + 1) {
                err = "There is no free node.";
                return false;
            }
            c = used++;
            Node& ch = pool[c];
            Node& par = pool[node];
            par.child[index] = c;
            ch.clear();
            ch.level = par.level + 1;
            ch.edge = par.edge * 0.5;
            int a = 1;
            real b = 2.0;
            for(int k = 0; k < 3; ++k) {
                ch.center[k] = par.center[k] + ((index & a) * b - 1.0) * par.edge * 0.25;
                a <<= 1;
                b *= 0.5;
            }
        }
        Node& ch = pool[c];
        ch.num++;
        ch.mass += s.f[SPHGPU_F_MASS][p];
        for(int k = 0; k < 3; ++k) ch.mcenter[k] += pos[k] * s.f[SPHGPU_F_MASS][p];
        next[p] = ch.first;
        ch.first = p;
        return true;
    }

    // BHNode::create_tree (src/bhtree.cpp:154-204)
    bool create(int node, const State& s)
    {
        std::fill(pool[node].child, pool[node].child + 8, -1);
        int p = pool[node].first;
        while(p >= 0) {
            const int pn = next[p];
            if(!assign(node, p, s)) return false;
            p = pn;
        }
        for(int i = 0; i < 8; ++i) {
            const int c = pool[node].child[i];
            if(c < 0) continue;
            if(pool[c].num > leaf_num && pool[node].level < max_level) {
                pool[c].mass = 0.0;
                pool[c].mcenter[0] = pool[c].mcenter[1] = pool[c].mcenter[2] = 0.0;
                if(!create(c, s)) return false;
            } else {
                pool[c].is_leaf = true;
                if(pool[c].mass > 0.0) {
                    for(int k = 0; k < 3; ++k) pool[c].mcenter[k] /= pool[c].mass;
                }
            }
            pool[node].mass += pool[c].mass;
            for(int k = 0; k < 3; ++k) pool[node].mcenter[k] += pool[c].mcenter[k] * pool[c].mass;
        }
        if(pool[node].mass > 0.0) {
            for(int k = 0; k < 3; ++k) pool[node].mcenter[k] /= pool[node].mass;
        }
        return true;
    }

    // BHTree::make (src/bhtree.cpp:59-115)
    bool make(const State& s, const Periodic& per)
    {
        const int n = s.n;
        if((int)pool.size() != 5 * n + 2) pool.assign(5 * n + 2, Node());
        Node& root = pool[0];
        root.first = -1;
        root.mass = 0.0;
        root.num = 0;
        root.mcenter[0] = root.mcenter[1] = root.mcenter[2] = 0.0;
        root.kernel_size = 0.0;
        root.is_leaf = false;
        root.level = 1;
        used = 1;
        if(n == 0) return true;
        if(per.valid) {
            real l = 0.0;
            for(int k = 0; k < 3; ++k) {
                root.center[k] = (per.hi[k] + per.lo[k]) * 0.5;
                const real r = per.hi[k] - per.lo[k];
                if(l < r) l = r;
            }
            root.edge = l;
        } else {
            real mn[3], mx[3];
            for(int k = 0; k < 3; ++k) {
                mn[k] = std::numeric_limits<real>::max();
                mx[k] = std::numeric_limits<real>::lowest();
            }
            for(int i = 0; i < n; ++i) {
                for(int k = 0; k < 3; ++k) {
                    const real x = s.f[SPHGPU_F_POS_X + k][i];
                    if(mn[k] > x) mn[k] = x;
                    if(mx[k] < x) mx[k] = x;
                }
            }
            // with more than one OpenMP thread the reference reduces over
            // per-thread slots that (except thread 0's) start at 0.0
            // (include/openmp.hpp:16-27, src/bhtree.cpp:68-91)
            if(root_origin) {
                for(int k = 0; k < 3; ++k) {
                    if(mn[k] > 0.0) mn[k] = 0.0;
                    if(mx[k] < 0.0) mx[k] = 0.0;
                }
            }
            real l = 0.0;
            for(int k = 0; k < 3; ++k) {
                root.center[k] = (mx[k] + mn[k]) * 0.5;
                const real r = mx[k] - mn[k];
                if(l < r) l = r;
            }
            root.edge = l;
        }
        next.assign(n, -1);
        for(int i = 0; i < n - 1; ++i) next[i] = i + 1;
        next[n - 1] = -1;
        root.first = 0;
        // the pool holds 5N nodes plus the root; allow one over like the
        // reference's `remaind < 0` check (src/bhtree.cpp:222)
        built = create(0, s);
        return built;
    }

    // BHNode::set_kernel (src/bhtree.cpp:249-275)
    real set_kernel(int node, const State& s)
    {
        Node& nd = pool[node];
        real k = 0.0;
        if(nd.is_leaf) {
            for(int p = nd.first; p >= 0; p = next[p]) {
                const real h = s.f[SPHGPU_F_SML][p];
                if(h > k) k = h;
            }
        } else {
            for(int i = 0; i < 8; ++i) {
                if(nd.child[i] >= 0) {
                    const real h = set_kernel(nd.child[i], s);
                    if(h > k) k = h;
                }
            }
        }
        pool[node].kernel_size = k;
        return k;
    }

    // BHNode::neighbor_search (src/bhtree.cpp:277-316); appends raw ids.
    void search(int node, const State& s, const Periodic& per, V3 ri, real hi, bool is_ij,
                std::vector<int>& out) const
    {
        const Node& nd = pool[node];
        const real h = is_ij ? std::max(hi, nd.kernel_size) : hi;
        const real h2 = h * h;
        const real l2 = sqr(nd.edge * 0.5 + h);
        const V3 d = per.rij(ri, {nd.center[0], nd.center[1], nd.center[2]});
        real m = sqr(d.x);
        if(sqr(d.y) > m) m = sqr(d.y);
        if(sqr(d.z) > m) m = sqr(d.z);
        if(m > l2) return;
        if(nd.is_leaf) {
            for(int p = nd.first; p >= 0; p = next[p]) {
                const V3 r = per.rij(ri, s.pos(p));
                if(dot(r, r) < h2) out.push_back(p);
            }
        } else {
            for(int i = 0; i < 8; ++i) {
                if(nd.child[i] >= 0) search(nd.child[i], s, per, ri, hi, is_ij, out);
            }
        }
    }
};

// Hernquist & Katz (1989) softened potential / force kernels
// (src/bhtree.cpp:318-345).
inline real hk_f(real r, real h)
{
    const real e = h * 0.5;
    const real u = r / e;
    if(u < 1.0) return (-0.5 * u * u * (1.0 / 3.0 - 3.0 / 20 * u * u + u * u * u / 20) + 1.4) / e;
    if(u < 2.0) return -1.0 / (15 * r) + (-u * u * (4.0 / 3.0 - u + 0.3 * u * u - u * u * u / 30) + 1.6) / e;
    return 1 / r;
}
inline real hk_g(real r, real h)
{
    const real e = h * 0.5;
    const real u = r / e;
    if(u < 1.0) return (4.0 / 3.0 - 1.2 * u * u + 0.5 * u * u * u) / (e * e * e);
    if(u < 2.0)
        return (-1.0 / 15 + 8.0 / 3 * u * u * u - 3 * u * u * u * u + 1.2 * u * u * u * u * u - u * u * u * u * u * u / 6.0)
            / (r * r * r);
    return 1 / (r * r * r);
}

// ---------------------------------------------------------------- Riemann
// van Leer limiter (src/gsph/g_fluid_force.cpp:32-41)
inline real limiter(real dq1, real dq2)
{
    const real p = dq1 * dq2;
    if(p <= 0) return 0.0;
    return 2.0 * p / (dq1 + dq2);
}

// HLL (src/gsph/g_fluid_force.cpp:173-204). state = (u, rho, p, c)
inline void riemann_hll(const real* L, const real* R, real& pstar, real& vstar)
{
    const real rl = std::sqrt(L[1]), rr = std::sqrt(R[1]);
    const real inv = 1.0 / (rl + rr);
    const real ut = (rl * L[0] + rr * R[0]) * inv;
    const real ct = (rl * L[3] + rr * R[3]) * inv;
    const real sl = std::min(L[0] - L[3], ut - ct);
    const real sr = std::max(R[0] + R[3], ut + ct);
    const real c1 = L[1] * (sl - L[0]);
    const real c2 = R[1] * (sr - R[0]);
    const real c3 = 1.0 / (c1 - c2);
    const real c4 = L[2] - L[0] * c1;
    const real c5 = R[2] - R[0] * c2;
    vstar = (c5 - c4) * c3;
    pstar = (c1 * c5 - c2 * c4) * c3;
}

// van Leer two-shock Newton solver (src/gsph/g_fluid_force.cpp:209-304).
// Returns the number of Newton iterations taken.
inline int riemann_iterative(const real* L, const real* R, real gamma, real& pstar, real& vstar)
{
    const real ul = L[0], rhol = L[1], pl = L[2];
    const real ur = R[0], rhor = R[1], pr = R[2];
    if(rhol < 0.0 || rhor < 0.0 || pl < 0.0 || pr < 0.0) {
        pstar = 0.0;
        vstar = 0.0;
        return 0;
    }
    const real g2 = 1.0 + gamma;
    const real g1 = 0.5 * g2 / gamma;
    const real smallp = 1e-25;
    const real vl = 1.0 / rhol, vr = 1.0 / rhor;
    const real cl = std::sqrt(gamma * pl * rhol);
    const real cr = std::sqrt(gamma * pr * rhor);
    real p = pr - pl - cr * (ur - ul);
    p = pl + p * cl / (cl + cr);
    p = std::max(p, smallp);
    int it = 0;
    for(; it < 20;) {
        const real pold = p;
        real wl = 1.0 + g1 * (p - pl) / pl;
        wl = cl * std::sqrt(wl);
        real wr = 1.0 + g1 * (p - pr) / pr;
        wr = cr * std::sqrt(wr);
        real zl = 4.0 * vl * wl * wl;
        zl = -zl * wl / (zl - g2 * (p - pl));
        real zr = 4.0 * vr * wr * wr;
        zr = zr * wr / (zr - g2 * (p - pr));
        const real usl = ul - (p - pl) / wl;
        const real usr = ur + (p - pr) / wr;
        p = p + (usr - usl) * (zl * zr) / (zr - zl);
        p = std::max(smallp, p);
        ++it;
        if(std::abs(p - pold) / p < 1e-6) break;
    }
    real wl = 1.0 + g1 * (p - pl) / pl;
    wl = cl * std::sqrt(wl);
    real wr = 1.0 + g1 * (p - pr) / pr;
    wr = cr * std::sqrt(wr);
    const real usl = ul - (p - pl) / wl;
    const real usr = ur + (p - pr) / wr;
    pstar = p;
    vstar = 0.5 * (usl + usr);
    return it;
}

// ---------------------------------------------------------------- solver
struct Oracle {
    sphgpu_params prm;
    State s;
    Periodic per;
    Kernel ker;
    Tree tree;
    real time = 0.0, dt = 0.0, h_per_v_sig = 0.0;
    bool first_pre = true;
    bool exhaustive = false;  // -DEXHAUSTIVE_SEARCH behaviour
    bool sr_failed = false;   // a primitive recovery in predict / correct did not converge
    int64_t newton_nonconv = 0, riemann_solves = 0, riemann_iters = 0;
    std::string err;

    int nngb() const { return prm.neighbor_number; }

    // per-particle gather/symmetric list, distance-sorted (src/bhtree.cpp:122-144
    // or src/exhaustive_search.cpp:11-42)
    bool neighbors(int i, bool is_ij, real hsearch, std::vector<int>& out)
    {
        out.clear();
        const V3 ri = s.pos(i);
        if(exhaustive) {
            const real k2 = hsearch * hsearch;
            for(int j = 0; j < s.n; ++j) {
                const V3 r = per.rij(ri, s.pos(j));
                const real r2 = dot(r, r);
                const real hj = s.f[SPHGPU_F_SML][j];
                const real lim = is_ij ? std::max(k2, hj * hj) : k2;
                if(r2 < lim) out.push_back(j);
            }
        } else {
            tree.search(0, s, per, ri, hsearch, is_ij, out);
        }
        if((int64_t)out.size() > (int64_t)nngb() * 1000) {
            err = "Neighbor list overflow";
            return false;
        }
        std::sort(out.begin(), out.end(), [&](int a, int b) {
            const V3 ra = per.rij(ri, s.pos(a));
            const V3 rb = per.rij(ri, s.pos(b));
            return dot(ra, ra) < dot(rb, rb);
        });
        return true;
    }

    static constexpr real A3 = 4.0 * M_PI / 3.0;

    // PreInteraction::initial_smoothing (src/pre_interaction.cpp:171-215)
    bool initial_smoothing()
    {
        bool ok = true;
#pragma omp parallel for schedule(dynamic, 64)
        for(int i = 0; i < s.n; ++i) {
            std::vector<int> list;
            real& h = s.f[SPHGPU_F_SML][i];
            h = std::pow(nngb() * s.f[SPHGPU_F_MASS][i] / (s.f[SPHGPU_F_DENS][i] * A3), 1.0 / 3);
            if(!neighbors(i, false, h, list)) {
                ok = false;
                continue;
            }
            const V3 ri = s.pos(i);
            real d = 0.0;
            for(int j : list) {
                const real r = norm(per.rij(ri, s.pos(j)));
                if(r >= h) break;
                d += s.f[SPHGPU_F_MASS][j] * ker.w(r, h);
            }
            s.f[SPHGPU_F_DENS][i] = d;
        }
        return ok;
    }

    // PreInteraction::newton_raphson (src/pre_interaction.cpp:227-283) and the
    // DISPH number-density variant (src/disph/d_pre_interaction.cpp:174-230).
    real newton(int i, const std::vector<int>& list, real ratio, bool disph, bool& conv)
    {
        real h = s.f[SPHGPU_F_SML][i] / ratio;
        const real b = disph ? nngb() / A3 : s.f[SPHGPU_F_MASS][i] * nngb() / A3;
        const V3 ri = s.pos(i);
        conv = true;
        for(int it = 0; it < 10; ++it) {
            const real hb = h;
            real d = 0.0, dd = 0.0;
            for(int j : list) {
                const real r = norm(per.rij(ri, s.pos(j)));
                if(r >= h) break;
                if(disph) {
                    d += ker.w(r, h);
                    dd += ker.dhw(r, h);
                } else {
                    d += s.f[SPHGPU_F_MASS][j] * ker.w(r, h);
                    dd += s.f[SPHGPU_F_MASS][j] * ker.dhw(r, h);
                }
            }
            const real f = d * pow3(h) - b;
            const real df = dd * pow3(h) + 3 * d * (h * h);
            h -= f / df;
            if(std::abs(h - hb) < (h + hb) * 1e-4) return h;
        }
        conv = false;
        return s.f[SPHGPU_F_SML][i] / ratio;
    }

    // PreInteraction::calculation for ssph (src/pre_interaction.cpp:39-169),
    // disph (src/disph/d_pre_interaction.cpp:21-162), gsph
    // (src/gsph/g_pre_interaction.cpp:27-144) and gdisph
    // (src/gdisph/gd_pre_interaction.cpp:29-198: the disph smoothing length,
    // density and pressure, the gsph gradients, its own AV switches).
    bool pre_interaction()
    {
        if(prm.sph_type == SPHGPU_SRGSPH) return sr_pre();
        if(first_pre) {
            if(!initial_smoothing()) return false;
            first_pre = false;
        }
        const int type = prm.sph_type;
        const bool gdisph = type == SPHGPU_GDISPH;
        const bool disph = type == SPHGPU_DISPH || gdisph, gsph = type == SPHGPU_GSPH;
        const real ratio = prm.iterative_sml ? 1.2 : 1.0;
        const real gamma = prm.gamma;
        real hvs = std::numeric_limits<real>::max();
        bool ok = true;
        int64_t nonconv = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(min : hvs) reduction(+ : nonconv)
        for(int i = 0; i < s.n; ++i) {
            std::vector<int> list;
            real& sml = s.f[SPHGPU_F_SML][i];
            const real mi = s.f[SPHGPU_F_MASS][i];
            sml = std::pow(nngb() * mi / (s.f[SPHGPU_F_DENS][i] * A3), 1.0 / 3) * ratio;
            if(!neighbors(i, false, sml, list)) {
                ok = false;
                continue;
            }
            if(prm.iterative_sml) {
                bool conv;
                sml = newton(i, list, ratio, disph, conv);
                if(!conv) ++nonconv;
            }
            const V3 ri = s.pos(i), vi = s.vel(i);
            const real ci = s.f[SPHGPU_F_SOUND][i];
            real dens = 0.0, dhd = 0.0, pres = 0.0, dhp = 0.0, ni = 0.0, dhn = 0.0;
            real vsig = ci * 2.0;
            int nn = 0;
            for(int j : list) {
                const V3 r = per.rij(ri, s.pos(j));
                const real rr = norm(r);
                if(rr >= sml) break;
                ++nn;
                const real mj = s.f[SPHGPU_F_MASS][j];
                if(disph) {
                    const real w = ker.w(rr, sml), dh = ker.dhw(rr, sml);
                    const real uj = s.f[SPHGPU_F_ENE][j];
                    dens += mj * w;
                    ni += w;
                    pres += mj * uj * w;
                    dhp += mj * uj * dh;
                    dhn += dh;
                } else {
                    dens += mj * ker.w(rr, sml);
                    if(!gsph) dhd += mj * ker.dhw(rr, sml);
                }
                if(i != j) {
                    const real v = ci + s.f[SPHGPU_F_SOUND][j] - 3.0 * dot(r, vi - s.vel(j)) / rr;
                    if(v > vsig) vsig = v;
                }
            }
            s.f[SPHGPU_F_DENS][i] = dens;
            if(disph) {
                s.f[SPHGPU_F_PRES][i] = (gamma - 1.0) * pres;
                s.f[SPHGPU_F_GRADH][i] = sml / (3 * ni) * dhp / (1.0 + sml / (3 * ni) * dhn);
            } else {
                s.f[SPHGPU_F_PRES][i] = (gamma - 1.0) * dens * s.f[SPHGPU_F_ENE][i];
                if(!gsph) s.f[SPHGPU_F_GRADH][i] = 1.0 / (1.0 + sml / (3 * dens) * dhd);
            }
            s.neighbor[i] = nn;
            const real hv = sml / vsig;
            if(hv < hvs) hvs = hv;

            if((gsph || gdisph) && prm.gsph_2nd_order) {
                // MUSCL gradients (src/gsph/g_pre_interaction.cpp:112-136,
                // src/gdisph/gd_pre_interaction.cpp:119-139)
                V3 dd{0, 0, 0}, du{0, 0, 0}, dv[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                const real ui = s.f[SPHGPU_F_ENE][i];
                for(int n = 0; n < nn; ++n) {
                    const int j = list[n];
                    const V3 r = per.rij(ri, s.pos(j));
                    const real rr = norm(r);
                    const V3 dw = ker.dw(r, rr, sml);
                    const real mj = s.f[SPHGPU_F_MASS][j];
                    dd = dd + dw * mj;
                    du = du + dw * (mj * (s.f[SPHGPU_F_ENE][j] - ui));
                    const V3 vj = s.vel(j);
                    dv[0] = dv[0] + dw * (mj * (vj.x - vi.x));
                    dv[1] = dv[1] + dw * (mj * (vj.y - vi.y));
                    dv[2] = dv[2] + dw * (mj * (vj.z - vi.z));
                }
                s.set_grad(0, i, dd);
                s.set_grad(1, i, (dd * ui + du) * (gamma - 1.0));
                const real rinv = 1.0 / s.f[SPHGPU_F_DENS][i];
                for(int k = 0; k < 3; ++k) s.set_grad(2 + k, i, dv[k] * rinv);
            }
            if(gsph) continue;

            // artificial viscosity switches (src/pre_interaction.cpp:115-161,
            // src/disph/d_pre_interaction.cpp:106-154; gdisph's Balsara switch
            // weights by mass and normalises by density, its implicit alpha
            // update weights by mass x energy, src/gdisph/gd_pre_interaction.cpp:141-195)
            const real hi = sml;
            real& alpha = s.f[SPHGPU_F_ALPHA][i];
            if(prm.use_balsara_switch) {
                real divv = 0.0;
                V3 rot{0, 0, 0};
                for(int n = 0; n < nn; ++n) {
                    const int j = list[n];
                    const V3 r = per.rij(ri, s.pos(j));
                    const real rr = norm(r);
                    const V3 dw = ker.dw(r, rr, hi);
                    const V3 vij = vi - s.vel(j);
                    const real wgt = (disph && !gdisph) ? s.f[SPHGPU_F_MASS][j] * s.f[SPHGPU_F_ENE][j]
                                                        : s.f[SPHGPU_F_MASS][j];
                    divv -= wgt * dot(vij, dw);
                    rot = rot + cross(vij, dw) * wgt;
                }
                if(disph && !gdisph) {
                    const real pinv = (gamma - 1.0) / s.f[SPHGPU_F_PRES][i];
                    divv *= pinv;
                    rot = rot * pinv;
                } else {
                    divv /= s.f[SPHGPU_F_DENS][i];
                    rot = {rot.x / s.f[SPHGPU_F_DENS][i], rot.y / s.f[SPHGPU_F_DENS][i], rot.z / s.f[SPHGPU_F_DENS][i]};
                }
                s.f[SPHGPU_F_BALSARA][i] = std::abs(divv) / (std::abs(divv) + norm(rot) + 1e-4 * ci / hi);
                if(prm.use_time_dependent_av) {
                    const real tau = prm.epsilon_av * ci / hi;
                    const real da = (-(alpha - prm.alpha_min) * tau + std::max(-divv, (real)0.0) * (prm.alpha_max - alpha)) * dt;
                    alpha += da;
                }
            } else if(prm.use_time_dependent_av) {
                real divv = 0.0;
                for(int n = 0; n < nn; ++n) {
                    const int j = list[n];
                    const V3 r = per.rij(ri, s.pos(j));
                    const real rr = norm(r);
                    const V3 dw = ker.dw(r, rr, hi);
                    const V3 vij = vi - s.vel(j);
                    const real wgt = disph ? s.f[SPHGPU_F_MASS][j] * s.f[SPHGPU_F_ENE][j] : s.f[SPHGPU_F_MASS][j];
                    divv -= wgt * dot(vij, dw);
                }
                if(disph) divv *= (gamma - 1.0) / s.f[SPHGPU_F_PRES][i];
                else divv /= s.f[SPHGPU_F_DENS][i];
                const real tau = prm.epsilon_av * ci / hi;
                const real si = std::max(-divv, (real)0.0);
                alpha = (alpha + dt * tau * prm.alpha_min + si * dt * prm.alpha_max) / (1.0 + dt * tau + si * dt);
            }
        }
        newton_nonconv += nonconv;
        h_per_v_sig = hvs;
        if(!exhaustive && ok) tree.set_kernel(0, s);
        return ok;
    }

    // Monaghan (1997) AV (src/fluid_force.cpp:88-106)
    real av(int i, int j, V3 rij) const
    {
        const V3 vij = s.vel(i) - s.vel(j);
        const real vr = dot(vij, rij);
        if(vr < 0) {
            const real alpha = 0.5 * (s.f[SPHGPU_F_ALPHA][i] + s.f[SPHGPU_F_ALPHA][j]);
            const real bal = 0.5 * (s.f[SPHGPU_F_BALSARA][i] + s.f[SPHGPU_F_BALSARA][j]);
            const real w = vr / norm(rij);
            const real vsig = s.f[SPHGPU_F_SOUND][i] + s.f[SPHGPU_F_SOUND][j] - 3.0 * w;
            const real rinv = 2.0 / (s.f[SPHGPU_F_DENS][i] + s.f[SPHGPU_F_DENS][j]);
            return -0.5 * bal * alpha * vsig * w * rinv;
        }
        return 0;
    }
    // Artificial conductivity (src/fluid_force.cpp:108-116)
    real ac(int i, int j, V3 rij, V3 dwij) const
    {
        const real vsig = prm.use_gravity
            ? std::abs(dot(s.vel(i) - s.vel(j), rij) / norm(rij))
            : std::sqrt(2.0 * std::abs(s.f[SPHGPU_F_PRES][i] - s.f[SPHGPU_F_PRES][j]) / (s.f[SPHGPU_F_DENS][i] + s.f[SPHGPU_F_DENS][j]));
        return prm.alpha_ac * s.f[SPHGPU_F_MASS][j] * vsig * (s.f[SPHGPU_F_ENE][i] - s.f[SPHGPU_F_ENE][j]) * dot(dwij, rij) / norm(rij);
    }

    // FluidForce::calculation for ssph (src/fluid_force.cpp:26-86), disph
    // (src/disph/d_fluid_force.cpp:26-86), gsph (src/gsph/g_fluid_force.cpp:44-171)
    // and gdisph (src/gdisph/gd_fluid_force.cpp:45-178: the gsph MUSCL states
    // and HLL star pressure inside the disph pressure-energy terms)
    bool fluid_force()
    {
        if(prm.sph_type == SPHGPU_SRGSPH) return sr_force();
        const int type = prm.sph_type;
        bool ok = true;
        int64_t solves = 0, iters = 0;
        std::vector<real> ax(s.n), ay(s.n), az(s.n), de(s.n);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : solves, iters)
        for(int i = 0; i < s.n; ++i) {
            std::vector<int> list;
            if(!neighbors(i, true, s.f[SPHGPU_F_SML][i], list)) {
                ok = false;
                continue;
            }
            const V3 ri = s.pos(i), vi = s.vel(i);
            const real hi = s.f[SPHGPU_F_SML][i];
            const real mi = s.f[SPHGPU_F_MASS][i], ui = s.f[SPHGPU_F_ENE][i];
            const real Pi = s.f[SPHGPU_F_PRES][i], rhoi = s.f[SPHGPU_F_DENS][i];
            const real gi = s.f[SPHGPU_F_GRADH][i];
            V3 acc{0, 0, 0};
            real dene = 0.0;
            for(int j : list) {
                const V3 r = per.rij(ri, s.pos(j));
                const real rr = norm(r);
                const real hj = s.f[SPHGPU_F_SML][j];
                if(rr >= std::max(hi, hj) || rr == 0.0) continue;
                const V3 vj = s.vel(j);
                const real mj = s.f[SPHGPU_F_MASS][j];
                const V3 dwi = ker.dw(r, rr, hi);
                const V3 dwj = ker.dw(r, rr, hj);
                real pstar = 0.0, vstar = 0.0;
                V3 e{0, 0, 0};
                if(type == SPHGPU_GSPH || type == SPHGPU_GDISPH) {
                    const real rinv = 1.0 / rr;
                    e = r * rinv;
                    const real vei = dot(vi, e), vej = dot(vj, e);
                    real L[4], R[4];
                    if(prm.gsph_2nd_order) {
                        const real di = 0.5 * (1.0 - s.f[SPHGPU_F_SOUND][i] * dt * rinv);
                        const real dj = 0.5 * (1.0 - s.f[SPHGPU_F_SOUND][j] * dt * rinv);
                        const real dvij = vei - vej;
                        V3 gvi, gvj;
                        gvi.x = dot(s.grad(2, i), e);
                        gvi.y = dot(s.grad(3, i), e);
                        gvi.z = dot(s.grad(4, i), e);
                        gvj.x = dot(s.grad(2, j), e);
                        gvj.y = dot(s.grad(3, j), e);
                        gvj.z = dot(s.grad(4, j), e);
                        const real dvei = dot(gvi, e) * rr, dvej = dot(gvj, e) * rr;
                        R[0] = vei - limiter(dvij, dvei) * di;
                        L[0] = vej + limiter(dvij, dvej) * dj;
                        const real rhoj = s.f[SPHGPU_F_DENS][j];
                        const real ddij = rhoi - rhoj;
                        const real ddi = dot(s.grad(0, i), e) * rr, ddj = dot(s.grad(0, j), e) * rr;
                        R[1] = rhoi - limiter(ddij, ddi) * di;
                        L[1] = rhoj + limiter(ddij, ddj) * dj;
                        const real Pj = s.f[SPHGPU_F_PRES][j];
                        const real dpij = Pi - Pj;
                        const real dpi = dot(s.grad(1, i), e) * rr, dpj = dot(s.grad(1, j), e) * rr;
                        R[2] = Pi - limiter(dpij, dpi) * di;
                        L[2] = Pj + limiter(dpij, dpj) * dj;
                        R[3] = std::sqrt(prm.gamma * R[2] / R[1]);
                        L[3] = std::sqrt(prm.gamma * L[2] / L[1]);
                    } else {
                        R[0] = vei; R[1] = rhoi; R[2] = Pi; R[3] = s.f[SPHGPU_F_SOUND][i];
                        L[0] = vej; L[1] = s.f[SPHGPU_F_DENS][j]; L[2] = s.f[SPHGPU_F_PRES][j]; L[3] = s.f[SPHGPU_F_SOUND][j];
                    }
                    if(type == SPHGPU_GSPH && prm.riemann_solver == SPHGPU_RIEMANN_ITERATIVE) {
                        iters += riemann_iterative(L, R, prm.gamma, pstar, vstar);
                        ++solves;
                    } else {
                        riemann_hll(L, R, pstar, vstar);
                    }
                }
                if(type == SPHGPU_GSPH) {
                    const V3 vij = e * vstar;
                    const real r2i = 1.0 / sqr(rhoi);
                    const real r2j = 1.0 / sqr(s.f[SPHGPU_F_DENS][j]);
                    const V3 f = dwi * (mj * pstar * r2i) + dwj * (mj * pstar * r2j);
                    acc = acc - f;
                    dene -= dot(f, vij - vi);
                    continue;
                }
                const V3 dwij = (dwi + dwj) * 0.5;
                const V3 vij = vi - vj;
                const real pij = av(i, j, r);
                const real dac = prm.use_ac ? ac(i, j, r, dwij) : 0.0;
                if(type == SPHGPU_DISPH) {
                    const real g2u = sqr(prm.gamma - 1.0) * ui;
                    const real g2up = g2u / Pi;
                    const real muinv = 1.0 / (mi * ui);
                    const real uj = s.f[SPHGPU_F_ENE][j];
                    const real fij = 1.0 - gi / (mj * uj);
                    const real fji = 1.0 - s.f[SPHGPU_F_GRADH][j] * muinv;
                    const real upj = uj / s.f[SPHGPU_F_PRES][j];
                    acc = acc - (dwi * (mj * (g2up * uj * fij + 0.5 * pij)) + dwj * (mj * (g2u * upj * fji + 0.5 * pij)));
                    dene += mj * g2up * uj * fij * dot(vij, dwi) + 0.5 * mj * pij * dot(vij, dwij) + dac;
                } else if(type == SPHGPU_GDISPH) {
                    const real g2u = sqr(prm.gamma - 1.0) * ui;
                    const real g2up = g2u / Pi;
                    const real muinv = 1.0 / (mi * ui);
                    const real uj = s.f[SPHGPU_F_ENE][j];
                    const real Pj = s.f[SPHGPU_F_PRES][j];
                    const real fij = 1.0 - gi / (mj * uj);
                    const real fji = 1.0 - s.f[SPHGPU_F_GRADH][j] * muinv;
                    const real upj = uj / Pj;
                    const real psi = pstar / Pi, psj = pstar / Pj;
                    acc = acc - (dwi * (mj * (g2up * uj * fij * psi + 0.5 * pij))
                                 + dwj * (mj * (g2u * upj * fji * psj + 0.5 * pij)));
                    dene += mj * g2up * uj * fij * psi * dot(vij, dwi) + 0.5 * mj * pij * dot(vij, dwij) + dac;
                } else {
                    const real ppr = Pi / sqr(rhoi);
                    const real pj = s.f[SPHGPU_F_PRES][j] / sqr(s.f[SPHGPU_F_DENS][j]);
                    acc = acc - (dwi * (mj * (ppr * gi + 0.5 * pij)) + dwj * (mj * (pj * s.f[SPHGPU_F_GRADH][j] + 0.5 * pij)));
                    dene += mj * ppr * gi * dot(vij, dwi) + 0.5 * mj * pij * dot(vij, dwij) + dac;
                }
            }
            ax[i] = acc.x;
            ay[i] = acc.y;
            az[i] = acc.z;
            de[i] = dene;
        }
        riemann_solves += solves;
        riemann_iters += iters;
        if(!ok) return false;
        s.f[SPHGPU_F_ACC_X] = ax;
        s.f[SPHGPU_F_ACC_Y] = ay;
        s.f[SPHGPU_F_ACC_Z] = az;
        s.f[SPHGPU_F_DENE] = de;
        return true;
    }

    // BHNode::calc_force (src/bhtree.cpp:347-393)
    void tree_force(int node, int i, V3 ri, real hi, real theta2, real G, V3& acc, real& phi) const
    {
        const Node& nd = tree.pool[node];
        const real l2 = nd.edge * nd.edge;
        const V3 d = per.rij(ri, {nd.mcenter[0], nd.mcenter[1], nd.mcenter[2]});
        const real d2 = dot(d, d);
        if(l2 > theta2 * d2 || d2 < l2) {
            if(nd.is_leaf) {
                for(int p = nd.first; p >= 0; p = tree.next[p]) {
                    if(p == i) continue;
                    const V3 r = per.rij(ri, s.pos(p));
                    const real rr = norm(r);
                    const real mp = s.f[SPHGPU_F_MASS][p], hp = s.f[SPHGPU_F_SML][p];
                    phi -= G * mp * (hk_f(rr, hi) + hk_f(rr, hp)) * 0.5;
                    const real c = G * mp * (hk_g(rr, hi) + hk_g(rr, hp)) * 0.5;
                    acc = acc - r * c;
                }
            } else {
                for(int c = 0; c < 8; ++c) {
                    if(nd.child[c] >= 0) tree_force(nd.child[c], i, ri, hi, theta2, G, acc, phi);
                }
            }
        } else {
            const real rinv = 1.0 / std::sqrt(d2);
            phi -= G * nd.mass * rinv;
            acc = acc - d * (G * nd.mass * pow3(rinv));
        }
    }

    // GravityForce::calculation (src/gravity_force.cpp:52-89); direct=true is
    // the -DEXHAUSTIVE_SEARCH branch.
    bool gravity(bool direct)
    {
        if(!prm.use_gravity) return true;
        const real G = prm.g_constant, theta2 = prm.theta * prm.theta;
#pragma omp parallel for schedule(dynamic, 64)
        for(int i = 0; i < s.n; ++i) {
            V3 acc = s.acc(i);
            real phi = 0.0;
            const V3 ri = s.pos(i);
            const real hi = s.f[SPHGPU_F_SML][i];
            if(direct) {
                V3 force{0, 0, 0};
                for(int j = 0; j < s.n; ++j) {
                    const V3 r = per.rij(ri, s.pos(j));
                    const real rr = norm(r);
                    const real mj = s.f[SPHGPU_F_MASS][j], hj = s.f[SPHGPU_F_SML][j];
                    phi -= G * mj * (hk_f(rr, hi) + hk_f(rr, hj)) * 0.5;
                    force = force - r * (G * mj * (hk_g(rr, hi) + hk_g(rr, hj)) * 0.5);
                }
                acc = acc + force;
            } else {
                tree_force(0, i, ri, hi, theta2, G, acc, phi);
            }
            s.f[SPHGPU_F_ACC_X][i] = acc.x;
            s.f[SPHGPU_F_ACC_Y][i] = acc.y;
            s.f[SPHGPU_F_ACC_Z][i] = acc.z;
            s.f[SPHGPU_F_PHI][i] = phi;
        }
        return true;
    }

    // TimeStep::calculation (src/timestep.cpp:18-38)
    void timestep()
    {
        if(prm.sph_type == SPHGPU_SRGSPH) return sr_timestep();
        real dtmin = std::numeric_limits<real>::max();
        for(int i = 0; i < s.n; ++i) {
            const real a = norm(s.acc(i));
            if(a > 0.0) {
                const real d = prm.cfl_force * std::sqrt(s.f[SPHGPU_F_SML][i] / a);
                if(d < dtmin) dtmin = d;
            }
        }
        dt = std::min(prm.cfl_sound * h_per_v_sig, dtmin);
    }

    // Solver::predict (src/solver.cpp:1046-1061)
    void predict()
    {
        if(prm.sph_type == SPHGPU_SRGSPH) return sr_predict();
        const real cs = prm.gamma * (prm.gamma - 1.0);
        for(int i = 0; i < s.n; ++i) {
            for(int k = 0; k < 3; ++k) {
                real& v = s.f[SPHGPU_F_VEL_X + k][i];
                real& vp = s.f[SPHGPU_F_VELP_X + k][i];
                const real a = s.f[SPHGPU_F_ACC_X + k][i];
                vp = v + a * (0.5 * dt);
            }
            s.f[SPHGPU_F_ENE_P][i] = s.f[SPHGPU_F_ENE][i] + s.f[SPHGPU_F_DENE][i] * (0.5 * dt);
            for(int k = 0; k < 3; ++k) {
                s.f[SPHGPU_F_POS_X + k][i] += s.f[SPHGPU_F_VELP_X + k][i] * dt;
                s.f[SPHGPU_F_VEL_X + k][i] += s.f[SPHGPU_F_ACC_X + k][i] * dt;
            }
            s.f[SPHGPU_F_ENE][i] += s.f[SPHGPU_F_DENE][i] * dt;
            s.f[SPHGPU_F_SOUND][i] = std::sqrt(cs * s.f[SPHGPU_F_ENE][i]);
            for(int k = 0; k < 3; ++k) per.apply(s.f[SPHGPU_F_POS_X + k][i], k);
        }
    }

    // Solver::correct (src/solver.cpp:1104-1112)
    void correct()
    {
        if(prm.sph_type == SPHGPU_SRGSPH) return sr_correct();
        const real cs = prm.gamma * (prm.gamma - 1.0);
        for(int i = 0; i < s.n; ++i) {
            for(int k = 0; k < 3; ++k) {
                s.f[SPHGPU_F_VEL_X + k][i] = s.f[SPHGPU_F_VELP_X + k][i] + s.f[SPHGPU_F_ACC_X + k][i] * (0.5 * dt);
            }
            s.f[SPHGPU_F_ENE][i] = s.f[SPHGPU_F_ENE_P][i] + s.f[SPHGPU_F_DENE][i] * (0.5 * dt);
            s.f[SPHGPU_F_SOUND][i] = std::sqrt(cs * s.f[SPHGPU_F_ENE][i]);
        }
    }

    // ------------------------------------------------------------ SRGSPH
    // Special-relativistic GSPH (src/srgsph/*.cpp; Kitajima, Inutsuka & Seno
    // 2025).  Conserved state per particle: S (canonical momentum), e
    // (canonical energy), N (lab-frame baryon density), nu (baryons); the
    // primitives follow from PrimitiveRecovery.
    struct SRPrim {
        V3 vel;
        real density, pressure, sound, enthalpy, gamma_lor;
    };

    V3 sr_S(int i) const { return {s.f[SPHGPU_F_SR_S_X][i], s.f[SPHGPU_F_SR_S_Y][i], s.f[SPHGPU_F_SR_S_Z][i]}; }
    V3 sr_dS(int i) const { return {s.f[SPHGPU_F_SR_DS_X][i], s.f[SPHGPU_F_SR_DS_Y][i], s.f[SPHGPU_F_SR_DS_Z][i]}; }

    // PrimitiveRecovery::solve_lorentz_factor (src/srgsph/sr_primitive_recovery.cpp:23-76):
    // Newton on (g^2-1)(X e g - 1)^2 - S^2 (X g^2 - 1)^2 / c^2 = 0, X = G/(G-1).
    bool sr_lorentz(real S_mag, real e, real& g) const
    {
        const real ge = prm.gamma, c = prm.sr_c_speed;
        const real X = ge / (ge - 1.0);
        const real c2 = c * c;
        const real S2 = S_mag * S_mag;
        g = 1.0 + std::sqrt(1.0 + S2 / c2) / X;
        for(int it = 0; it < 100; ++it) {
            const real g2 = g * g;
            const real g2m1 = g2 - 1.0;
            const real xe = X * e * g - 1.0;
            const real xg = X * g2 - 1.0;
            const real f = g2m1 * xe * xe - S2 * xg * xg / c2;
            const real df = 2.0 * g * xe * xe + 2.0 * g2m1 * xe * X * e - 2.0 * S2 * xg * 2.0 * X * g / c2;
            const real delta = f / df;
            g -= delta;
            if(g < 1.0) g = 1.0 + 1.0e-10;
            if(std::abs(delta) < 1.0e-10 * g) return true;
        }
        return false;
    }

    // PrimitiveRecovery::conserved_to_primitive (src/srgsph/sr_primitive_recovery.cpp:82-160)
    bool sr_c2p(V3 S, real e, real N, SRPrim& o) const
    {
        const real ge = prm.gamma, c = prm.sr_c_speed;
        const real S_mag = norm(S);
        if(!sr_lorentz(S_mag, e, o.gamma_lor)) return false;
        const real X = ge / (ge - 1.0);
        const real g = o.gamma_lor, g2 = g * g;
        const real num = X * g2 - 1.0;
        const real den = g * (X * e * g - 1.0);
        o.vel = S * (num / den);
        o.density = N / g;
        const real v_mag = norm(o.vel);
        const real c2 = c * c;
        if(v_mag > 1.0e-10) o.enthalpy = S_mag / (g * v_mag);
        else o.enthalpy = 1.0 + (e - 1.0) / c2;
        o.pressure = (ge - 1.0) * o.density * c2 * (o.enthalpy - 1.0) / ge;
        o.sound = std::sqrt((ge - 1.0) * (o.enthalpy - 1.0) / o.enthalpy);
        return true;
    }

    // srgsph::PreInteraction::compute_smoothing_length
    // (src/srgsph/sr_pre_interaction.cpp:103-246): damped fixed point
    // h <- (h + eta Vp*(C_smooth h)^(1/3)) / 2 over the list members.
    real sr_smoothing_length(int i, const std::vector<int>& list) const
    {
        real h = s.f[SPHGPU_F_SML][i];
        const V3 ri = s.pos(i);
        for(int iter = 0; iter < 20; ++iter) {
            const real hs = prm.sr_c_smooth * h;
            real sum = 0.0;
            for(int j : list) {
                const real r = norm(per.rij(ri, s.pos(j)));
                if(r < hs) sum += ker.w(r, hs);
            }
            sum += ker.w(0.0, hs);
            if(sum < 1.0e-20) {
                h *= 1.5;
                continue;
            }
            const real vp = 1.0 / sum;
            const real hn = prm.sr_eta * std::pow(vp, 1.0 / real(3));
            const real hd = 0.5 * (h + hn);
            if(std::abs(hd - h) < 1.0e-6 * h) return hd;
            h = hd;
            if(h < 1.0e-10) h = 1.0e-10;
            if(h > 10.0) h = 10.0;
        }
        return h;
    }

    // srgsph::PreInteraction::calculation (src/srgsph/sr_pre_interaction.cpp:248-407).
    // The reference updates N inside its particle loop while the same loop
    // reads the neighbours' N, so the result depends on the loop order; this
    // restatement runs the loop serially in index order (the reference's
    // single-thread result).
    bool sr_pre()
    {
        if(first_pre) {
            // initial_smoothing (src/srgsph/sr_pre_interaction.cpp:31-67)
            for(int i = 0; i < s.n; ++i)
                s.f[SPHGPU_F_SML][i] = prm.sr_eta * std::pow(s.f[SPHGPU_F_SR_NU][i] / s.f[SPHGPU_F_SR_N][i], 1.0 / 3);
            first_pre = false;
        }
        std::vector<int> list;
        for(int i = 0; i < s.n; ++i) {
            if(!neighbors(i, false, s.f[SPHGPU_F_SML][i], list)) return false;
            real& sml = s.f[SPHGPU_F_SML][i];
            const real nu_i = s.f[SPHGPU_F_SR_NU][i];
            if(prm.iterative_sml) sml = sr_smoothing_length(i, list);
            else sml = prm.sr_eta * std::pow(nu_i / s.f[SPHGPU_F_SR_N][i], 1.0 / 3);
            const real h = sml;
            const V3 ri = s.pos(i);
            // compute_volume (src/srgsph/sr_pre_interaction.cpp:69-101)
            real sw = 0.0;
            for(int j : list) {
                const real r = norm(per.rij(ri, s.pos(j)));
                if(r < h) sw += ker.w(r, h);
            }
            sw += ker.w(0.0, h);
            const real vp = 1.0 / sw;
            s.f[SPHGPU_F_SR_N][i] = nu_i / vp;
            SRPrim pi;
            if(!sr_c2p(sr_S(i), s.f[SPHGPU_F_SR_E][i], s.f[SPHGPU_F_SR_N][i], pi)) {
                err = "Lorentz factor solver did not converge";
                return false;
            }
            s.f[SPHGPU_F_VEL_X][i] = pi.vel.x;
            s.f[SPHGPU_F_VEL_Y][i] = pi.vel.y;
            s.f[SPHGPU_F_VEL_Z][i] = pi.vel.z;
            s.f[SPHGPU_F_PRES][i] = pi.pressure;
            s.f[SPHGPU_F_DENS][i] = pi.density;
            s.f[SPHGPU_F_SOUND][i] = pi.sound;
            s.f[SPHGPU_F_SR_GAMMA_LOR][i] = pi.gamma_lor;
            s.f[SPHGPU_F_SR_ENTHALPY][i] = pi.enthalpy;
            V3 gd{0, 0, 0}, gp{0, 0, 0}, gv[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            real omega = 0.0;
            for(int j : list) {
                const V3 r = per.rij(ri, s.pos(j));
                const real rr = norm(r);
                if(rr >= h || rr == 0.0) continue;
                SRPrim pj;
                if(!sr_c2p(sr_S(j), s.f[SPHGPU_F_SR_E][j], s.f[SPHGPU_F_SR_N][j], pj)) {
                    err = "Lorentz factor solver did not converge";
                    return false;
                }
                const V3 dw = ker.dw(r, rr, h);
                const real vol_j = s.f[SPHGPU_F_SR_NU][j] / s.f[SPHGPU_F_SR_N][j];
                omega += vol_j * ker.w(rr, h);
                gd = gd + dw * (vol_j * (pj.density - pi.density));
                gp = gp + dw * (vol_j * (pj.pressure - pi.pressure));
                gv[0] = gv[0] + dw * (vol_j * (pj.vel.x - pi.vel.x));
                gv[1] = gv[1] + dw * (vol_j * (pj.vel.y - pi.vel.y));
                gv[2] = gv[2] + dw * (vol_j * (pj.vel.z - pi.vel.z));
            }
            if(omega > 0.0) {
                const real oi = 1.0 / omega;
                s.set_grad(0, i, gd * oi);
                s.set_grad(1, i, gp * oi);
                for(int k = 0; k < 3; ++k) s.set_grad(2 + k, i, gv[k] * oi);
            } else {
                for(int g = 0; g < 5; ++g) s.set_grad(g, i, V3{0, 0, 0});
            }
        }
        return true;
    }

    // FluidForce::compute_shock_velocity (src/srgsph/sr_fluid_force.cpp:366-420):
    // Taub adiabat and Rankine-Hugoniot (Pons, Marti & Mueller 2000).
    real sr_shock_velocity(real p_a, real rho_a, real h_a, real vx_a, real W_a, real p_b, bool left) const
    {
        const real ge = prm.gamma;
        const real dp = p_a - p_b;
        const real A = 1.0 + (ge - 1.0) * dp / (ge * p_b);
        const real B = -h_a * dp / (ge * p_b);
        const real Cc = -h_a * h_a + h_a * dp / rho_a;
        const real disc = B * B - 4.0 * A * Cc;
        if(disc < 0.0) return vx_a;
        const real h_b = (-B + std::sqrt(disc)) / (2.0 * A);
        const real rho_b = ge * p_b / ((ge - 1.0) * (h_b - 1.0));
        const real hra = h_a / rho_a;
        const real hrb = h_b / rho_b;
        const real j2 = -(p_b - p_a) / (hrb - hra);
        if(j2 < 0.0) return vx_a;
        const real j = left ? -std::sqrt(j2) : std::sqrt(j2);
        const real rwa = rho_a * W_a;
        const real rwa2 = rwa * rwa;
        const real numer = rwa2 * vx_a + j * std::sqrt(j2 + rwa2 * (1.0 - vx_a * vx_a));
        const real denom = rwa2 + j2;
        const real Vs = numer / denom;
        const real Ws = 1.0 / std::sqrt(1.0 - Vs * Vs);
        const real t1 = h_a * W_a * vx_a + Ws * (p_b - p_a) / j + Ws * Vs / (rho_a * W_a);
        const real t2 = h_a * W_a + (p_b - p_a) / j;
        return t2 / t1;
    }

    // FluidForce::compute_rarefaction_velocity (src/srgsph/sr_fluid_force.cpp:436-480):
    // 100 explicit Euler steps of dv/dp along the isentrope.
    real sr_rarefaction_velocity(real p_a, real rho_a, real vx_a, real p_b, bool left) const
    {
        const real ge = prm.gamma;
        const real dp = (p_b - p_a) / 100;
        real p = p_a, vx = vx_a;
        for(int k = 0; k < 100; ++k) {
            const real eps = (ge - 1.0) * p / rho_a;
            const real rho = rho_a * std::pow(p / p_a, 1.0 / ge);
            const real h = 1.0 + eps + p / rho;
            const real cs = std::sqrt(ge * p / (rho * h));
            const real W = 1.0 / std::sqrt(1.0 - vx * vx);
            const real sign = left ? -1.0 : 1.0;
            const real dvdp = sign / (rho * h * W * W * cs);
            vx += dvdp * dp;
            p += dp;
            if(vx >= 1.0) vx = 0.99999;
            if(vx <= -1.0) vx = -0.99999;
        }
        return vx;
    }

    real sr_wave(real p_star, real p_a, real rho_a, real h_a, real vx_a, real W_a, bool left) const
    {
        return p_star > p_a ? sr_shock_velocity(p_a, rho_a, h_a, vx_a, W_a, p_star, left)
                            : sr_rarefaction_velocity(p_a, rho_a, vx_a, p_star, left);
    }

    // FluidForce::exact_riemann_solver (src/srgsph/sr_fluid_force.cpp:236-350).
    // state = (v, n, P, c_s)
    void sr_riemann(const real* L, const real* R, real& pstar, real& vstar) const
    {
        const real ge = prm.gamma;
        const real vL = L[0], nL = L[1], pL = L[2];
        const real vR = R[0], nR = R[1], pR = R[2];
        const real hL = 1.0 + ge * pL / ((ge - 1.0) * nL);
        const real hR = 1.0 + ge * pR / ((ge - 1.0) * nR);
        const real WL = 1.0 / std::sqrt(1.0 - vL * vL);
        const real WR = 1.0 / std::sqrt(1.0 - vR * vR);
        real ps = 0.5 * (pL + pR);
        for(int it = 0; it < 50; ++it) {
            const real vLs = sr_wave(ps, pL, nL, hL, vL, WL, true);
            const real vRs = sr_wave(ps, pR, nR, hR, vR, WR, false);
            const real f = vRs - vLs;
            if(std::abs(f) < 1.0e-8) {
                pstar = ps;
                vstar = 0.5 * (vLs + vRs);
                return;
            }
            const real dp = ps * 1.0e-6;
            const real vLp = sr_wave(ps + dp, pL, nL, hL, vL, WL, true);
            const real vRp = sr_wave(ps + dp, pR, nR, hR, vR, WR, false);
            const real fp = vRp - vLp;
            const real df = (fp - f) / dp;
            if(std::abs(df) > 1.0e-12) {
                real pn = ps - 0.5 * f / df;
                pn = std::max(pn, 0.01 * std::min(pL, pR));
                ps = pn;
            } else if(f > 0) {
                ps *= 0.9;
            } else {
                ps *= 1.1;
            }
        }
        const real vLs = sr_wave(ps, pL, nL, hL, vL, WL, true);
        const real vRs = sr_wave(ps, pR, nR, hR, vR, WR, false);
        pstar = ps;
        vstar = 0.5 * (vLs + vRs);
    }

    // srgsph::FluidForce::calculation (src/srgsph/sr_fluid_force.cpp:47-232)
    bool sr_force()
    {
        bool ok = true;
        const real ge = prm.gamma;
#pragma omp parallel for schedule(dynamic, 64)
        for(int i = 0; i < s.n; ++i) {
            std::vector<int> list;
            if(!neighbors(i, true, s.f[SPHGPU_F_SML][i], list)) {
                ok = false;
                continue;
            }
            const V3 ri = s.pos(i), vi = s.vel(i);
            const real hi = s.f[SPHGPU_F_SML][i], nu_i = s.f[SPHGPU_F_SR_NU][i];
            const real ci = s.f[SPHGPU_F_SOUND][i], Pi = s.f[SPHGPU_F_PRES][i];
            const real Ni = s.f[SPHGPU_F_SR_N][i], gi = s.f[SPHGPU_F_SR_GAMMA_LOR][i];
            V3 dS{0, 0, 0};
            real de = 0.0;
            for(int j : list) {
                const V3 r = per.rij(ri, s.pos(j));
                const real rr = norm(r);
                const real hj = s.f[SPHGPU_F_SML][j];
                if(rr >= std::max(hi, hj) || rr == 0.0) continue;
                const real rinv = 1.0 / rr;
                const V3 e = r * rinv;
                const V3 vj = s.vel(j);
                const real vei = dot(vi, e), vej = dot(vj, e);
                const real cj = s.f[SPHGPU_F_SOUND][j], Pj = s.f[SPHGPU_F_PRES][j];
                const real Nj = s.f[SPHGPU_F_SR_N][j], gj = s.f[SPHGPU_F_SR_GAMMA_LOR][j];
                const real n_i = Ni / gi, n_j = Nj / gj;
                real right[4], left[4], pstar, vstar;
                bool first = !prm.sr_2nd_order;
                if(prm.sr_2nd_order) {
                    const real di = 0.5 * (1.0 - ci * dt * rinv);
                    const real dj = 0.5 * (1.0 - cj * dt * rinv);
                    const real dv = vei - vej;
                    const V3 dvi{dot(s.grad(2, i), e), dot(s.grad(3, i), e), dot(s.grad(4, i), e)};
                    const V3 dvj{dot(s.grad(2, j), e), dot(s.grad(3, j), e), dot(s.grad(4, j), e)};
                    const real dve_i = dot(dvi, e) * rr;
                    const real dve_j = dot(dvj, e) * rr;
                    const real min_cs = std::min(ci, cj);
                    const real shock = prm.sr_c_shock * std::abs(vei - vej);
                    const real pjump = std::abs(std::log10(Pi / Pj));
                    if((shock > min_cs) || (pjump > prm.sr_c_cd)) {
                        first = true;
                    } else {
                        right[0] = vei - limiter(dv, dve_i) * di;
                        left[0] = vej + limiter(dv, dve_j) * dj;
                        const real dn = n_i - n_j;
                        const real dn_i = dot(s.grad(0, i), e) * rr / gi;
                        const real dn_j = dot(s.grad(0, j), e) * rr / gj;
                        right[1] = n_i - limiter(dn, dn_i) * di;
                        left[1] = n_j + limiter(dn, dn_j) * dj;
                        const real dpp = Pi - Pj;
                        const real dp_i = dot(s.grad(1, i), e) * rr;
                        const real dp_j = dot(s.grad(1, j), e) * rr;
                        right[2] = Pi - limiter(dpp, dp_i) * di;
                        left[2] = Pj + limiter(dpp, dp_j) * dj;
                        right[3] = std::sqrt(ge * right[2] / right[1]);
                        left[3] = std::sqrt(ge * left[2] / left[1]);
                    }
                }
                if(first) {
                    right[0] = vei;
                    right[1] = n_i;
                    right[2] = Pi;
                    right[3] = ci;
                    left[0] = vej;
                    left[1] = n_j;
                    left[2] = Pj;
                    left[3] = cj;
                }
                sr_riemann(left, right, pstar, vstar);
                const V3 dwi = ker.dw(r, rr, 2.0 * hi);
                const V3 dwj = ker.dw(r, rr, 2.0 * hj);
                const V3 dwij = dwi - dwj;
                const real Vi = nu_i / Ni;
                const real Vj = s.f[SPHGPU_F_SR_NU][j] / Nj;
                const real V2 = 0.5 * (Vi * Vi + Vj * Vj);
                dS = dS - dwij * (pstar * V2);
                const V3 vij = e * vstar;
                de -= dot(vij, dwij) * (pstar * V2);
            }
            s.f[SPHGPU_F_SR_DS_X][i] = dS.x / nu_i;
            s.f[SPHGPU_F_SR_DS_Y][i] = dS.y / nu_i;
            s.f[SPHGPU_F_SR_DS_Z][i] = dS.z / nu_i;
            s.f[SPHGPU_F_SR_DE][i] = de / nu_i;
        }
        return ok;
    }

    // srgsph::TimeStep::calculation (src/srgsph/sr_timestep.cpp:14-59)
    void sr_timestep()
    {
        real dmin = std::numeric_limits<real>::max();
        for(int i = 0; i < s.n; ++i) {
            const real cs = std::max(s.f[SPHGPU_F_SOUND][i], real(1.0e-10));
            const real d = prm.cfl_sound * s.f[SPHGPU_F_SML][i] / cs;
            if(d < dmin) dmin = d;
        }
        dt = dmin;
    }

    void sr_store(int i, const SRPrim& q)
    {
        s.f[SPHGPU_F_VEL_X][i] = q.vel.x;
        s.f[SPHGPU_F_VEL_Y][i] = q.vel.y;
        s.f[SPHGPU_F_VEL_Z][i] = q.vel.z;
        s.f[SPHGPU_F_ENE][i] = q.pressure / ((prm.gamma - 1.0) * q.density);
        s.f[SPHGPU_F_PRES][i] = q.pressure;
        s.f[SPHGPU_F_DENS][i] = q.density;
        s.f[SPHGPU_F_SOUND][i] = q.sound;
        s.f[SPHGPU_F_SR_GAMMA_LOR][i] = q.gamma_lor;
        s.f[SPHGPU_F_SR_ENTHALPY][i] = q.enthalpy;
    }

    // Solver::predict, SRGSPH branch (src/solver.cpp:992-1043)
    void sr_predict()
    {
        for(int i = 0; i < s.n; ++i) {
            const V3 S = sr_S(i), dS = sr_dS(i);
            real& e = s.f[SPHGPU_F_SR_E][i];
            const real de = s.f[SPHGPU_F_SR_DE][i];
            const V3 Sh = S + dS * (0.5 * dt);
            const real eh = e + de * (0.5 * dt);
            const V3 Sn = S + dS * dt;
            s.f[SPHGPU_F_SR_S_X][i] = Sn.x;
            s.f[SPHGPU_F_SR_S_Y][i] = Sn.y;
            s.f[SPHGPU_F_SR_S_Z][i] = Sn.z;
            e += de * dt;
            SRPrim ph, pf;
            if(!sr_c2p(Sh, eh, s.f[SPHGPU_F_SR_N][i], ph) || !sr_c2p(Sn, e, s.f[SPHGPU_F_SR_N][i], pf)) {
                sr_failed = true;
                continue;
            }
            s.f[SPHGPU_F_POS_X][i] += ph.vel.x * dt;
            s.f[SPHGPU_F_POS_Y][i] += ph.vel.y * dt;
            s.f[SPHGPU_F_POS_Z][i] += ph.vel.z * dt;
            for(int k = 0; k < 3; ++k) per.apply(s.f[SPHGPU_F_POS_X + k][i], k);
            sr_store(i, pf);
            s.f[SPHGPU_F_VELP_X][i] = ph.vel.x;
            s.f[SPHGPU_F_VELP_Y][i] = ph.vel.y;
            s.f[SPHGPU_F_VELP_Z][i] = ph.vel.z;
            s.f[SPHGPU_F_ENE_P][i] = ph.pressure / ((prm.gamma - 1.0) * ph.density);
        }
    }

    // Solver::correct, SRGSPH branch (src/solver.cpp:1075-1102)
    void sr_correct()
    {
        for(int i = 0; i < s.n; ++i) {
            const V3 dS = sr_dS(i);
            const real de = s.f[SPHGPU_F_SR_DE][i];
            const V3 Sh = sr_S(i) - dS * (0.5 * dt);
            const real eh = s.f[SPHGPU_F_SR_E][i] - de * (0.5 * dt);
            const V3 S = Sh + dS * (0.5 * dt);
            const real e = eh + de * (0.5 * dt);
            s.f[SPHGPU_F_SR_S_X][i] = S.x;
            s.f[SPHGPU_F_SR_S_Y][i] = S.y;
            s.f[SPHGPU_F_SR_S_Z][i] = S.z;
            s.f[SPHGPU_F_SR_E][i] = e;
            SRPrim q;
            if(!sr_c2p(S, e, s.f[SPHGPU_F_SR_N][i], q)) {
                sr_failed = true;
                continue;
            }
            sr_store(i, q);
        }
    }

    bool make_tree()
    {
        if(exhaustive) return true;
        if(!tree.make(s, per)) {
            err = tree.err;
            return false;
        }
        return true;
    }

    // Tail of Solver::initialize (src/solver.cpp:941-964)
    bool initialize()
    {
        const real cs = prm.gamma * (prm.gamma - 1.0);
        for(int i = 0; i < s.n; ++i) {
            s.f[SPHGPU_F_ALPHA][i] = prm.av_alpha;
            s.f[SPHGPU_F_BALSARA][i] = 1.0;
            s.f[SPHGPU_F_SOUND][i] = std::sqrt(cs * s.f[SPHGPU_F_ENE][i]);
        }
        return make_tree() && pre_interaction() && fluid_force() && gravity(exhaustive);
    }

    // Solver::integrate (src/solver.cpp:966-978) + update_time
    bool integrate()
    {
        timestep();
        predict();
        if(sr_failed) return err = "Lorentz factor solver did not converge", false;
        if(!make_tree() || !pre_interaction() || !fluid_force() || !gravity(exhaustive)) return false;
        correct();
        if(sr_failed) return err = "Lorentz factor solver did not converge", false;
        time += dt;
        return true;
    }

    // LaneEmdenData::get_theta / dtheta_dxi (src/relaxation/lane_emden_data.cpp:66-113):
    // linear interpolation in a table with ascending xi.
    static real table_at(const real* x, const real* y, int64_t np, real xi)
    {
        const real* it = std::lower_bound(x, x + np, xi);
        if(it == x + np) return 0.0;
        if(it == x) return y[0];
        const int64_t i1 = it - x, i0 = i1 - 1;
        const real frac = (xi - x[i0]) / (x[i1] - x[i0]);
        return y[i0] * (1.0 - frac) + y[i1] * frac;
    }

    // One step of the Lane-Emden relaxation loop (src/solver.cpp:779-829):
    // SPH forces, minus LaneEmdenRelaxation::compute_relaxation_force
    // (src/relaxation/lane_emden_relaxation.cpp:35-116), TimeStep dt x 0.1,
    // v = 0 and x += a dt^2 / 2.  `first` sets the sound speeds as the set-up
    // before the loop does (src/solver.cpp:744-752).
    bool relax_step(const real* tx, const real* tth, const real* tdth, int64_t np, real xi1, real alpha, real K,
                    bool first, real& dt_out)
    {
        if(first) {
            const real cs = prm.gamma * (prm.gamma - 1.0);
            for(int i = 0; i < s.n; ++i) s.f[SPHGPU_F_SOUND][i] = std::sqrt(cs * s.f[SPHGPU_F_ENE][i]);
        }
        if(!make_tree() || !pre_interaction() || !fluid_force() || !gravity(exhaustive)) return false;
        const real gamma = prm.gamma;
        for(int i = 0; i < s.n; ++i) {
            const V3 p = s.pos(i);
            const real r = norm(p);
            if(r < 1e-12) continue;
            const real xi = r / alpha;
            if(xi >= xi1) continue;
            const real theta = xi <= 0.0 ? 1.0 : table_at(tx, tth, np, xi);
            const real dtheta = xi <= 0.0 ? 0.0 : table_at(tx, tdth, np, xi);
            if(theta <= 0.0) continue;
            const real prefactor = K * gamma * 1.5 / alpha;
            const real a_r = -prefactor * std::pow(theta, gamma - 1.0) * dtheta;
            const real rinv = 1.0 / r;
            s.f[SPHGPU_F_ACC_X][i] -= -a_r * p.x * rinv;
            s.f[SPHGPU_F_ACC_Y][i] -= -a_r * p.y * rinv;
            s.f[SPHGPU_F_ACC_Z][i] -= -a_r * p.z * rinv;
        }
        timestep();
        const real d = dt * 0.1;
        for(int i = 0; i < s.n; ++i) {
            for(int k = 0; k < 3; ++k) {
                s.f[SPHGPU_F_VEL_X + k][i] = 0.0;
                real& x = s.f[SPHGPU_F_POS_X + k][i];
                x += 0.5 * s.f[SPHGPU_F_ACC_X + k][i] * d * d;
                per.apply(x, k);
            }
        }
        dt_out = d;
        return true;
    }
};

}  // namespace oracle

using oracle::Oracle;

extern "C" {

void* oracle_create(const sphgpu_params* p, int64_t n, const double* const* fields, int exhaustive)
{
    auto* o = new Oracle;
    o->prm = *p;
    o->exhaustive = exhaustive != 0;
    o->ker.type = p->kernel;
    o->per.valid = p->periodic != 0;
    for(int k = 0; k < 3; ++k) {
        o->per.lo[k] = p->range_min[k];
        o->per.hi[k] = p->range_max[k];
        o->per.range[k] = p->range_max[k] - p->range_min[k];
    }
    o->tree.max_level = p->max_tree_level;
    o->tree.root_origin = p->tree_root_origin != 0;
    o->tree.leaf_num = p->leaf_particle_num;
    o->s.n = (int)n;
    for(int k = 0; k < SPHGPU_NFIELDS; ++k) {
        o->s.f[k].assign(n, 0.0);
        if(fields && fields[k]) std::copy(fields[k], fields[k] + n, o->s.f[k].begin());
    }
    o->s.neighbor.assign(n, 0);
    return o;
}

void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }
const char* oracle_last_error(void* h) { return static_cast<Oracle*>(h)->err.c_str(); }

int oracle_get(void* h, double* const* fields)
{
    auto* o = static_cast<Oracle*>(h);
    for(int k = 0; k < SPHGPU_NFIELDS; ++k) {
        if(!fields[k]) continue;
        if(k == SPHGPU_F_NEIGHBOR) {
            for(int i = 0; i < o->s.n; ++i) fields[k][i] = o->s.neighbor[i];
        } else {
            std::copy(o->s.f[k].begin(), o->s.f[k].end(), fields[k]);
        }
    }
    return 0;
}

int oracle_set(void* h, const double* const* fields)
{
    auto* o = static_cast<Oracle*>(h);
    for(int k = 0; k < SPHGPU_NFIELDS; ++k) {
        if(fields[k] && k != SPHGPU_F_NEIGHBOR) std::copy(fields[k], fields[k] + o->s.n, o->s.f[k].begin());
    }
    return 0;
}

void oracle_set_dt(void* h, double dt) { static_cast<Oracle*>(h)->dt = dt; }
double oracle_get_dt(void* h) { return static_cast<Oracle*>(h)->dt; }
double oracle_get_time(void* h) { return static_cast<Oracle*>(h)->time; }
double oracle_get_h_per_v_sig(void* h) { return static_cast<Oracle*>(h)->h_per_v_sig; }
void oracle_set_first(void* h, int first) { static_cast<Oracle*>(h)->first_pre = first != 0; }

int oracle_tree_make(void* h) { return static_cast<Oracle*>(h)->make_tree() ? 0 : -1; }
int oracle_set_kernel(void* h)
{
    auto* o = static_cast<Oracle*>(h);
    o->tree.set_kernel(0, o->s);
    return 0;
}
int oracle_pre(void* h) { return static_cast<Oracle*>(h)->pre_interaction() ? 0 : -1; }
int oracle_force(void* h) { return static_cast<Oracle*>(h)->fluid_force() ? 0 : -1; }
int oracle_gravity(void* h, int direct) { return static_cast<Oracle*>(h)->gravity(direct != 0) ? 0 : -1; }
int oracle_timestep(void* h)
{
    static_cast<Oracle*>(h)->timestep();
    return 0;
}
int oracle_predict(void* h)
{
    static_cast<Oracle*>(h)->predict();
    return static_cast<Oracle*>(h)->sr_failed ? -1 : 0;
}
int oracle_correct(void* h)
{
    static_cast<Oracle*>(h)->correct();
    return static_cast<Oracle*>(h)->sr_failed ? -1 : 0;
}
int oracle_initialize(void* h) { return static_cast<Oracle*>(h)->initialize() ? 0 : -1; }
int oracle_integrate(void* h) { return static_cast<Oracle*>(h)->integrate() ? 0 : -1; }

int oracle_relax_step(void* h, const double* xi, const double* theta, const double* dtheta, int64_t np,
                      double xi_1, double alpha, double K, int first, double* dt_relax)
{
    return static_cast<Oracle*>(h)->relax_step(xi, theta, dtheta, np, xi_1, alpha, K, first != 0, *dt_relax) ? 0
                                                                                                             : -1;
}

void oracle_energies(void* h, double* K, double* U, double* W, double* mom)
{
    auto* o = static_cast<Oracle*>(h);
    double k = 0, u = 0, w = 0, px = 0, py = 0, pz = 0;
    for(int i = 0; i < o->s.n; ++i) {
        const double m = o->s.f[SPHGPU_F_MASS][i];
        const oracle::V3 v = o->s.vel(i);
        k += 0.5 * m * oracle::dot(v, v);
        u += m * o->s.f[SPHGPU_F_ENE][i];
        if(o->prm.use_gravity) w += 0.5 * m * o->s.f[SPHGPU_F_PHI][i];
        px += m * v.x;
        py += m * v.y;
        pz += m * v.z;
    }
    *K = k;
    *U = u;
    *W = w;
    if(mom) {
        mom[0] = px;
        mom[1] = py;
        mom[2] = pz;
    }
}

void oracle_counters(void* h, int64_t* out3)
{
    auto* o = static_cast<Oracle*>(h);
    out3[0] = o->newton_nonconv;
    out3[1] = o->riemann_solves;
    out3[2] = o->riemann_iters;
}

// Distance-sorted neighbour lists of every particle with radius sml
// (is_ij as in BHTree::neighbor_search). offsets[n+1]; ids may be NULL.
int oracle_neighbor_lists(void* h, int is_ij, int64_t* offsets, int32_t* ids, int64_t cap)
{
    auto* o = static_cast<Oracle*>(h);
    const int n = o->s.n;
    std::vector<std::vector<int>> lists(n);
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 64)
    for(int i = 0; i < n; ++i) {
        if(!o->neighbors(i, is_ij != 0, o->s.f[SPHGPU_F_SML][i], lists[i])) ok = false;
    }
    if(!ok) return -1;
    offsets[0] = 0;
    for(int i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + (int64_t)lists[i].size();
    if(!ids) return 0;
    if(offsets[n] > cap) return -1;
    for(int i = 0; i < n; ++i) std::copy(lists[i].begin(), lists[i].end(), ids + offsets[i]);
    return 0;
}

// Octree nodes in depth-first preorder (children in index order 0..7), for
// bitwise tree parity: per node level, is_leaf, num, and
// center[3], edge, mass, mcenter[3], kernel_size packed in dbl[9*k..].
int64_t oracle_tree_nodes(void* h, int32_t* ints /* [3*cap] */, double* dbl /* [9*cap] */, int64_t cap)
{
    auto* o = static_cast<Oracle*>(h);
    if(o->tree.used == 0) return 0;
    int64_t k = 0;
    std::vector<int> stack{0};
    while(!stack.empty()) {
        const int nd = stack.back();
        stack.pop_back();
        const auto& N = o->tree.pool[nd];
        if(k < cap && ints && dbl) {
            ints[3 * k] = N.level;
            ints[3 * k + 1] = N.is_leaf ? 1 : 0;
            ints[3 * k + 2] = N.num;
            double* d = dbl + 9 * k;
            d[0] = N.center[0]; d[1] = N.center[1]; d[2] = N.center[2]; d[3] = N.edge;
            d[4] = N.mass; d[5] = N.mcenter[0]; d[6] = N.mcenter[1]; d[7] = N.mcenter[2];
            d[8] = N.kernel_size;
        }
        ++k;
        if(!N.is_leaf) {
            for(int c = 7; c >= 0; --c) {
                if(N.child[c] >= 0) stack.push_back(N.child[c]);
            }
        }
    }
    return k;
}

// Kernel functions for the kernel-derivative tests (test/kernel_test/kernel_test.cpp).
double oracle_kernel_w(int type, double r, double h)
{
    oracle::Kernel k{type};
    return k.w(r, h);
}
double oracle_kernel_dwc(int type, double r, double h)
{
    oracle::Kernel k{type};
    return k.dwc(r, h);
}
double oracle_kernel_dhw(int type, double r, double h)
{
    oracle::Kernel k{type};
    return k.dhw(r, h);
}

// Pair-level Riemann solvers. state = (u, rho, p, c). Returns iterations.
int oracle_riemann(int solver, const double* left, const double* right, double gamma,
                   double* pstar, double* vstar)
{
    if(solver == SPHGPU_RIEMANN_ITERATIVE) return oracle::riemann_iterative(left, right, gamma, *pstar, *vstar);
    oracle::riemann_hll(left, right, *pstar, *vstar);
    return 0;
}

}  // extern "C"
