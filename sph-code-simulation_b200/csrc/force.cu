// force.cu — FluidForce::calculation for ssph, disph, gsph and gdisph.
//
// Reference: src/fluid_force.cpp:26-116 (ssph pair force, Monaghan-97
// artificial viscosity, artificial conductivity), src/disph/d_fluid_force.cpp:26-86
// (Hopkins-2013 pressure-energy force), src/gsph/g_fluid_force.cpp:32-304
// (van Leer limiter, MUSCL reconstruction, HLL and iterative Riemann solvers),
// src/gdisph/gd_fluid_force.cpp:45-228 (gdisph: the MUSCL states' HLL star
// pressure inside the disph pressure-energy terms).
//
// Gather form, no atomics: a group of G lanes owns particle i and strides over
// its symmetric list (the is_ij tree walk), skipping pairs with
// r >= max(h_i, h_j) or r == 0 exactly as the reference; acc and du/dt are
// accumulated in FP64 and group-reduced, then overwrite acc (the reference
// overwrites too; gravity adds afterwards).
// T = double: plain FP64 form.  T = float: pair arithmetic in FP32 with FP64
// accumulators (mixed form); the Riemann Newton iteration runs in FP32 and its
// final step in FP64.
#include <cfloat>
#include <cuda_runtime.h>

#include "context.cuh"
#include "mlp.cuh"
#include "scan_sort.cuh"

namespace sphgpu {

namespace {

constexpr int FBLK = 256;

template <typename T>
struct V3 {
    T x, y, z;
};

// van Leer (1979) limiter (src/gsph/g_fluid_force.cpp:32-41)
template <typename T>
__device__ __forceinline__ T limiter(T dq1, T dq2)
{
    const T p = dq1 * dq2;
    if(p <= T(0)) return T(0);
    return T(2) * p / (dq1 + dq2);
}

// HLL (src/gsph/g_fluid_force.cpp:173-204); state = (u, rho, p, c)
template <typename T>
__device__ __forceinline__ void riemann_hll(const T* L, const T* R, T& pstar, T& vstar)
{
    const T rl = sqrt(L[1]), rr = sqrt(R[1]);
    const T inv = T(1) / (rl + rr);
    const T ut = (rl * L[0] + rr * R[0]) * inv;
    const T ct = (rl * L[3] + rr * R[3]) * inv;
    const T sl = fmin(L[0] - L[3], ut - ct);
    const T sr = fmax(R[0] + R[3], ut + ct);
    const T c1 = L[1] * (sl - L[0]);
    const T c2 = R[1] * (sr - R[0]);
    const T c3 = T(1) / (c1 - c2);
    const T c4 = L[2] - L[0] * c1;
    const T c5 = R[2] - R[0] * c2;
    vstar = (c5 - c4) * c3;
    pstar = (c1 * c5 - c2 * c4) * c3;
}

// One van Leer two-shock Newton update of p (src/gsph/g_fluid_force.cpp:255-283).
template <typename T>
__device__ __forceinline__ T vl_newton_step(T p, T ul, T pl, T vl, T cl, T ur, T pr, T vr, T cr, T g1, T g2)
{
    T wl = T(1) + g1 * (p - pl) / pl;
    wl = cl * sqrt(wl);
    T wr = T(1) + g1 * (p - pr) / pr;
    wr = cr * sqrt(wr);
    T zl = T(4) * vl * wl * wl;
    zl = -zl * wl / (zl - g2 * (p - pl));
    T zr = T(4) * vr * wr * wr;
    zr = zr * wr / (zr - g2 * (p - pr));
    const T usl = ul - (p - pl) / wl;
    const T usr = ur + (p - pr) / wr;
    p = p + (usr - usl) * (zl * zr) / (zr - zl);
    return fmax(T(1e-25), p);
}

// Final wave speeds and u* at p (src/gsph/g_fluid_force.cpp:285-298), FP64.
__device__ __forceinline__ double vl_ustar(double p, double ul, double pl, double cl, double ur, double pr,
                                           double cr, double g1)
{
    double wl = 1.0 + g1 * (p - pl) / pl;
    wl = cl * sqrt(wl);
    double wr = 1.0 + g1 * (p - pr) / pr;
    wr = cr * sqrt(wr);
    const double usl = ul - (p - pl) / wl;
    const double usr = ur + (p - pr) / wr;
    return 0.5 * (usl + usr);
}

// Screen of the learned start: one Newton step from the reference's
// linearised guess (src/gsph/g_fluid_force.cpp:244-246).  Returns the relative
// change and the stepped pressure.  Kept out of line: the pair loops that call
// it are register-bound.
__device__ __noinline__ double learned_screen(double ul, double pl, double vl, double cl, double ur, double pr,
                                              double vr, double cr, double g1, double g2, double& q1)
{
    double q0 = pr - pl - cr * (ur - ul);
    q0 = fmax(pl + q0 * cl / (cl + cr), 1e-25);
    q1 = vl_newton_step<double>(q0, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
    return fabs(q1 - q0) / q1;
}

// The screen for states with positive densities and pressures: relative change
// `ch` and stepped pressure `q1`; the network's guess is needed when ch >= 1e-2.
__device__ __forceinline__ void pair_screen(const double* L, const double* R, double gamma, double& ch, double& q1)
{
    const double g2 = 1.0 + gamma, g1 = 0.5 * g2 / gamma;
    const double cl = sqrt(gamma * L[2] * L[1]), cr = sqrt(gamma * R[2] * R[1]);
    ch = learned_screen(L[0], L[2], 1.0 / L[1], cl, R[0], R[2], 1.0 / R[1], cr, g1, g2, q1);
}

// Iterative solver (src/gsph/g_fluid_force.cpp:209-304).  Plain form: FP64
// throughout.  Mixed form: iterations in T = float, then one FP64 Newton step
// and the FP64 u*.  With `learned` set, Newton starts from the screened start
// (below; y = the network's log(p_star / p_L), read only when the screen
// rejects the linearised start), runs at most `budget` iterations to a 1e-10
// relative change (in FP64) and falls back to the plain start on failure.
// A screen the caller already ran is passed as (scr_ch >= 0, scr_q1).
template <typename T>
__device__ void riemann_iterative(const double* L, const double* R, double gamma, bool learned, float y, int budget,
                                  double& pstar, double& vstar, int& iters, int& fallback, double scr_ch = -1.0,
                                  double scr_q1 = 0.0, double tol = 1e-6)
{
    const double ul = L[0], rhol = L[1], pl = L[2];
    const double ur = R[0], rhor = R[1], pr = R[2];
    iters = 0;
    fallback = 0;
    if(rhol < 0.0 || rhor < 0.0 || pl < 0.0 || pr < 0.0) {
        pstar = 0.0;
        vstar = 0.0;
        return;
    }
    const double g2 = 1.0 + gamma;
    const double g1 = 0.5 * g2 / gamma;
    const double vl = 1.0 / rhol, vr = 1.0 / rhor;
    const double cl = sqrt(gamma * pl * rhol);
    const double cr = sqrt(gamma * pr * rhor);
    double p;
    if(learned) {
        // Learned start.  Screen first with one Newton step from the
        // reference's linearised guess: when that step moves p by less than
        // 1 % the linearised start is already in Newton's quadratic range
        // (nearly equal states, the common case inside a flow) and is kept;
        // otherwise Newton restarts from the network's guess.  Either way
        // Newton runs to a 1e-10 relative change within `budget` iterations,
        // else the reference's solver takes over.
        double q1 = scr_q1;
        const double ch = scr_ch >= 0.0 ? scr_ch : learned_screen(ul, pl, vl, cl, ur, pr, vr, cr, g1, g2, q1);
        iters = 1;
        const double guess = pl * exp((double)y);
        p = (ch < 1e-2 || !(guess > 0.0 && guess < 1e300)) ? q1 : guess;
        bool ok = ch < 1e-10;
        for(int it = 0; !ok && it < budget; ++it) {
            const double pold = p;
            p = vl_newton_step<double>(p, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
            ++iters;
            if(fabs(p - pold) / p < 1e-10) ok = true;
        }
        if(ok) {
            pstar = p;
            vstar = vl_ustar(p, ul, pl, cl, ur, pr, cr, g1);
            return;
        }
        fallback = 1;
    }
    double pg = pr - pl - cr * (ur - ul);
    pg = pl + pg * cl / (cl + cr);
    pg = fmax(pg, 1e-25);
    // (after a failed learned start the counted iterations keep accumulating)
    if(sizeof(T) == sizeof(double)) {
        p = pg;
        for(int it = 0; it < 20; ++it) {
            const double pold = p;
            p = vl_newton_step<double>(p, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
            ++iters;
            if(fabs(p - pold) / p < tol) break;
        }
    } else {
        float pf = (float)pg;
        const float ulf = (float)ul, plf = (float)pl, vlf = (float)vl, clf = (float)cl;
        const float urf = (float)ur, prf = (float)pr, vrf = (float)vr, crf = (float)cr;
        const float g1f = (float)g1, g2f = (float)g2;
        for(int it = 0; it < 20; ++it) {
            const float pold = pf;
            pf = vl_newton_step<float>(pf, ulf, plf, vlf, clf, urf, prf, vrf, crf, g1f, g2f);
            ++iters;
            if(fabsf(pf - pold) / pf < 1e-6f) break;
        }
        // final Newton step in FP64 (more of them down to a tolerance below FP32's)
        p = vl_newton_step<double>((double)pf, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
        for(int it = 0; tol < 1e-6 && it < 20; ++it) {
            const double pold = p;
            p = vl_newton_step<double>(p, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
            ++iters;
            if(fabs(p - pold) / p < tol) break;
        }
    }
    pstar = p;
    vstar = vl_ustar(p, ul, pl, cl, ur, pr, cr, g1);
}

// MODE: 0 = force (optionally harvesting pair states); 3 = force with the
// learned guess, deferring the pairs whose linearised start the screen
// rejects (their features and pair slots go to the MlpPairs rows); 4 = the
// deferred pairs only, with the network's guess, added to acc.
// Minimum resident blocks per SM (caps registers; measured on B200): FP64
// disph 2 (27.2 -> 24.5 ms on the 8.78 M sphere), FP64 gdisph 3 (8.8 -> 7.7 ms
// on the 2 M tube), FP32 disph 3 (17.3 -> 16.0 ms, once the next pair's index
// is fetched ahead), gsph and the other FP32 forms 4 (gsph 18.8 -> 9.6 ms
// against 3), FP64 ssph 3.
template <typename T, int TYPE>
constexpr int force_min_blocks()
{
    if(sizeof(T) == sizeof(float) && TYPE == SPHGPU_DISPH) return 3;
    if(sizeof(T) == sizeof(float) || TYPE == SPHGPU_GSPH) return 4;
    return TYPE == SPHGPU_DISPH ? 2 : 3;
}

// The particles a launch computes: all n, or (sub.idx != null) the listed
// ones (the mixed form's FP64 re-evaluation).  count = 0: the launch adds to
// no work or Riemann counter (the pairs were counted by the first pass).
struct Subset {
    const int* idx;
    int n;
    int count;
};

template <typename T, int G, int TYPE, int MODE>
__global__ void __launch_bounds__(FBLK, (force_min_blocks<T, TYPE>())) k_force(DevParams P, DevState S, int n, const int* __restrict__ list,
                                                const int* __restrict__ count, int cap, const double* __restrict__ dtp,
                                                DevStatus* __restrict__ st, MlpPairs mp, Harvest hv,
                                                float* __restrict__ accabs, Subset sub)
{
    constexpr int GPW = 32 / G;
    constexpr bool f32 = sizeof(T) == sizeof(float);
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * FBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * FBLK) >> 5;
    const double dt = *dtp;
    const double gamma = P.gamma;
    unsigned long long solves = 0, iters = 0, fallbacks = 0;
    unsigned n_cand = 0, n_pairs = 0;  // work counters of this lane
    const int nloop = sub.idx ? sub.n : n;

    for(long long wb = warp * GPW; wb < nloop; wb += nwarps * GPW) {
        const int slot = (int)(wb + ((threadIdx.x & 31) / G));
        const bool valid = slot < nloop;
        const int i = sub.idx ? (valid ? sub.idx[slot] : n) : slot;
        const int cnt = valid ? (MODE == 4 ? mp.dcount[i] : min(count[i], cap)) : 0;
        if(MODE == 4 && !__any_sync(FULL_MASK, cnt > 0)) continue;
        const int* li = list + (size_t)(valid ? i : 0) * (size_t)cap;
        const double4 pi = valid ? S.pos[i] : make_double4(0, 0, 0, 0);
        const double4 vi = valid ? S.vel[i] : make_double4(0, 0, 0, 1);
        const double4 ti = valid ? S.thermo[i] : make_double4(1, 1, 1, 1);
        const double4 si = valid ? S.visc[i] : make_double4(0, 0, 1, 0);
        const double hi = vi.w;
        double4 gi0 = make_double4(0, 0, 0, 0), gi1 = gi0, gi2 = gi0, gi3 = gi0;
        if((TYPE == SPHGPU_GSPH || TYPE == SPHGPU_GDISPH) && P.gsph2 && valid) {
            gi0 = S.grad[i];
            gi1 = S.grad[(size_t)n + i];
            gi2 = S.grad[2 * (size_t)n + i];
            gi3 = S.grad[3 * (size_t)n + i];
        }
        const T rhoi = (T)ti.x, Pi = (T)ti.y, ui = (T)ti.z, ci = (T)ti.w;
        const T mi = (T)pi.w;
        const KernH<T> khi(P.kernel, (T)hi);
        // per-particle factors of the pair terms
        const T ppr = Pi / (rhoi * rhoi);                             // ssph P_i / rho_i^2
        const T g2u = ((T)gamma - T(1)) * ((T)gamma - T(1)) * ui;     // disph (gamma-1)^2 u_i
        const T g2up = g2u / Pi;
        const T mu_inv = T(1) / (mi * ui);
        const T r2i = T(1) / (rhoi * rhoi);
        double ax = 0, ay = 0, az = 0, de = 0;
        float sabs = 0.f;  // mixed form: sum of |FP32 force terms|, the rounding-error scale
        n_cand += lane < cnt ? (unsigned)((cnt - lane + G - 1) / G) : 0u;
        // the next pair's index is fetched one iteration ahead, so the
        // neighbour's loads do not wait on the list load
        int jn = MODE != 4 && lane < cnt ? __ldg(&li[lane]) : 0;
        for(int k = lane; k < cnt; k += G) {
            float yq = 0.f;
            int j;
            if(MODE == 4) {
                const int row = mp.dstart[i] + k;
                const int kk = (int)(mp.skeys[row] - (uint64_t)i * (uint64_t)cap);
                yq = mp.y[mp.svals[row]];
                j = li[kk];
            } else {
                j = jn;
                if(k + G < cnt) jn = __ldg(&li[k + G]);
            }
            const double4 pj = ldg4(&S.pos[j]);
            const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double4 vj = ldg4(&S.vel[j]);
            const double hj = vj.w;
            double r, rinv;
            if constexpr(f32) {
                // the set predicate in FP64 (exact), the distance in FP32
                const double r2 = abs2x(d);
                if(!root_lt(r2, hi < hj ? hj : hi) || r2 == 0.0) continue;
                const float r2f = (float)r2;
                const float rif = rsqrtf(r2f);
                r = (double)(r2f * rif);
                rinv = (double)rif;
                if(!(r > 0.0)) continue;  // r^2 below FP32's range: coincident for the force
            } else {
                r = sqrt(abs2x(d));
                if(r >= (hi < hj ? hj : hi) || r == 0.0) continue;
                rinv = 1.0 / r;
            }
            ++n_pairs;
            const double4 tj = ldg4(&S.thermo[j]);
            const T rT = (T)r;
            const T rinvT = (T)rinv;
            const V3<T> rv{(T)d.x, (T)d.y, (T)d.z};
            const KernH<T> khj(P.kernel, (T)hj);
            const T ci_ = khi.dwc(rT, rinvT);
            const T cj_ = khj.dwc(rT, rinvT);
            const V3<T> dwi{rv.x * ci_, rv.y * ci_, rv.z * ci_};
            const V3<T> dwj{rv.x * cj_, rv.y * cj_, rv.z * cj_};
            const T mj = (T)pj.w;
            const T rhoj = (T)tj.x, Pj = (T)tj.y, uj = (T)tj.z, cj = (T)tj.w;
            // gdisph: the HLL star pressure of the MUSCL states scales the disph
            // pressure terms below by p_star / P_i and p_star / P_j
            // (src/gdisph/gd_fluid_force.cpp:95-178)
            T psi = T(1), psj = T(1);
            if(TYPE == SPHGPU_GSPH || TYPE == SPHGPU_GDISPH) {
                const double ex = d.x * rinv, ey = d.y * rinv, ez = d.z * rinv;
                const double vei = vi.x * ex + vi.y * ey + vi.z * ez;
                const double vej = vj.x * ex + vj.y * ey + vj.z * ez;
                double Lst[4], Rst[4];
                if(P.gsph2) {
                    // MUSCL reconstruction (src/gsph/g_fluid_force.cpp:103-140)
                    const double4 gj0 = ldg4(&S.grad[j]), gj1 = ldg4(&S.grad[(size_t)n + j]);
                    const double4 gj2 = ldg4(&S.grad[2 * (size_t)n + j]), gj3 = ldg4(&S.grad[3 * (size_t)n + j]);
                    const T di = T(0.5) * (T(1) - ci * (T)dt * (T)rinv);
                    const T dj = T(0.5) * (T(1) - cj * (T)dt * (T)rinv);
                    const T exT = (T)ex, eyT = (T)ey, ezT = (T)ez;
                    // velocity: dv_i[k] = grad_v[k] . e, dve_i = dv_i . e * r
                    const T dvi0 = (T)gi1.z * exT + (T)gi1.w * eyT + (T)gi2.x * ezT;
                    const T dvi1 = (T)gi2.y * exT + (T)gi2.z * eyT + (T)gi2.w * ezT;
                    const T dvi2 = (T)gi3.x * exT + (T)gi3.y * eyT + (T)gi3.z * ezT;
                    const T dvj0 = (T)gj1.z * exT + (T)gj1.w * eyT + (T)gj2.x * ezT;
                    const T dvj1 = (T)gj2.y * exT + (T)gj2.z * eyT + (T)gj2.w * ezT;
                    const T dvj2 = (T)gj3.x * exT + (T)gj3.y * eyT + (T)gj3.z * ezT;
                    const T dve_i = (dvi0 * exT + dvi1 * eyT + dvi2 * ezT) * rT;
                    const T dve_j = (dvj0 * exT + dvj1 * eyT + dvj2 * ezT) * rT;
                    const T dv_ij = (T)vei - (T)vej;
                    Rst[0] = (double)((T)vei - limiter(dv_ij, dve_i) * di);
                    Lst[0] = (double)((T)vej + limiter(dv_ij, dve_j) * dj);
                    const T dd_ij = rhoi - rhoj;
                    const T dd_i = ((T)gi0.x * exT + (T)gi0.y * eyT + (T)gi0.z * ezT) * rT;
                    const T dd_j = ((T)gj0.x * exT + (T)gj0.y * eyT + (T)gj0.z * ezT) * rT;
                    Rst[1] = (double)(rhoi - limiter(dd_ij, dd_i) * di);
                    Lst[1] = (double)(rhoj + limiter(dd_ij, dd_j) * dj);
                    const T dp_ij = Pi - Pj;
                    const T dp_i = ((T)gi0.w * exT + (T)gi1.x * eyT + (T)gi1.y * ezT) * rT;
                    const T dp_j = ((T)gj0.w * exT + (T)gj1.x * eyT + (T)gj1.y * ezT) * rT;
                    Rst[2] = (double)(Pi - limiter(dp_ij, dp_i) * di);
                    Lst[2] = (double)(Pj + limiter(dp_ij, dp_j) * dj);
                    Rst[3] = (double)sqrt((T)gamma * (T)Rst[2] / (T)Rst[1]);
                    Lst[3] = (double)sqrt((T)gamma * (T)Lst[2] / (T)Lst[1]);
                } else {
                    Rst[0] = vei;
                    Rst[1] = ti.x;
                    Rst[2] = ti.y;
                    Rst[3] = ti.w;
                    Lst[0] = vej;
                    Lst[1] = tj.x;
                    Lst[2] = tj.y;
                    Lst[3] = tj.w;
                }
                if(TYPE == SPHGPU_GDISPH) {
                    double pg, vg;
                    if(sizeof(T) == sizeof(double)) {
                        riemann_hll<double>(Lst, Rst, pg, vg);
                    } else {
                        const float Lf[4] = {(float)Lst[0], (float)Lst[1], (float)Lst[2], (float)Lst[3]};
                        const float Rf[4] = {(float)Rst[0], (float)Rst[1], (float)Rst[2], (float)Rst[3]};
                        float ps, vs;
                        riemann_hll<float>(Lf, Rf, ps, vs);
                        pg = ps;
                    }
                    psi = (T)pg / Pi;
                    psj = (T)pg / Pj;
                }
                if constexpr(TYPE == SPHGPU_GSPH) {
                    const bool states_ok = Lst[1] > 0.0 && Rst[1] > 0.0 && Lst[2] > 0.0 && Rst[2] > 0.0;
                    double scr_ch = -1.0, scr_q1 = 0.0;
                    if(MODE == 3 && states_ok) pair_screen(Lst, Rst, gamma, scr_ch, scr_q1);
                    if(MODE == 3 && !(scr_ch < 1e-2) && states_ok) {
                        // deferred to the completion pass, which solves it from
                        // the network's guess; with the row list full the pair
                        // is solved here from the linearised start instead
                        const unsigned long long row = atomicAdd(mp.rows, 1ull);
                        if((long long)row < mp.rcap) {
                            float x[MLP_IN];
                            mlp_features(Lst, Rst, gamma, x);
                            mp.feat[row] = make_uint4(pack_bf16x2(x[0], x[1]), pack_bf16x2(x[2], x[3]),
                                                      pack_bf16x2(x[4], 0.f), 0u);
                            mp.keys[row] = (uint64_t)i * (uint64_t)cap + (uint64_t)k;
                            atomicAdd(&st->mlp_guesses, 1ull);
                            continue;
                        }
                    }
                    double pstar, vstar;
                    if(P.riemann == SPHGPU_RIEMANN_ITERATIVE) {
                        int it = 0, fb = 0;
                        // learned start: the linearised guess where the screen
                        // accepts it, else the network's (a NaN guess selects
                        // the linearised one)
                        const bool learned = (MODE == 3 || MODE == 4) && states_ok;
                        riemann_iterative<T>(Lst, Rst, gamma, learned, MODE == 4 ? yq : __int_as_float(0x7fc00000),
                                             P.mlp_max_newton, pstar, vstar, it, fb, scr_ch, scr_q1, P.riemann_tol);
                        ++solves;
                        iters += it;
                        fallbacks += fb;
                        if(MODE == 0 && hv.mod) {
                            unsigned hsh = (unsigned)i * 0x9E3779B1u ^ (unsigned)k * 0x85EBCA77u ^ hv.salt;
                            hsh ^= hsh >> 15;
                            hsh *= 0x2C1B3C6Du;
                            hsh ^= hsh >> 12;
                            if(hsh % hv.mod == 0) {
                                const unsigned long long slot = atomicAdd(hv.count, 1ull);
                                if((long long)slot < hv.cap) {
                                    double* o = hv.out + 8 * slot;
                                    o[0] = Lst[0];
                                    o[1] = Lst[1];
                                    o[2] = Lst[2];
                                    o[3] = Rst[0];
                                    o[4] = Rst[1];
                                    o[5] = Rst[2];
                                    o[6] = gamma;
                                    o[7] = pstar;
                                }
                            }
                        }
                    } else if(sizeof(T) == sizeof(double)) {
                        riemann_hll<double>(Lst, Rst, pstar, vstar);
                    } else {
                        const float Lf[4] = {(float)Lst[0], (float)Lst[1], (float)Lst[2], (float)Lst[3]};
                        const float Rf[4] = {(float)Rst[0], (float)Rst[1], (float)Rst[2], (float)Rst[3]};
                        float ps, vs;
                        riemann_hll<float>(Lf, Rf, ps, vs);
                        pstar = ps;
                        vstar = vs;
                    }
                    // f = dw_i m_j p* / rho_i^2 + dw_j m_j p* / rho_j^2 (src/gsph/g_fluid_force.cpp:158-165)
                    const T ps = (T)pstar;
                    const T fi = mj * ps * r2i;
                    const T fj = mj * ps * (T(1) / (rhoj * rhoj));
                    const double fx = (double)(dwi.x * fi + dwj.x * fj);
                    const double fy = (double)(dwi.y * fi + dwj.y * fj);
                    const double fz = (double)(dwi.z * fi + dwj.z * fj);
                    ax -= fx;
                    ay -= fy;
                    az -= fz;
                    if constexpr(f32) sabs += (float)(fabs(fx) + fabs(fy) + fabs(fz));
                    de -= fx * (ex * vstar - vi.x) + fy * (ey * vstar - vi.y) + fz * (ez * vstar - vi.z);
                    continue;
                }
            }
            const double4 sj = ldg4(&S.visc[j]);
            const V3<T> dwij{(dwi.x + dwj.x) * T(0.5), (dwi.y + dwj.y) * T(0.5), (dwi.z + dwj.z) * T(0.5)};
            const V3<T> vij{(T)(vi.x - vj.x), (T)(vi.y - vj.y), (T)(vi.z - vj.z)};
            // artificial viscosity (src/fluid_force.cpp:88-106)
            T pij = 0;
            const T vr = vij.x * rv.x + vij.y * rv.y + vij.z * rv.z;
            if(vr < T(0)) {
                const T alpha = T(0.5) * ((T)si.x + (T)sj.x);
                const T bal = T(0.5) * ((T)si.y + (T)sj.y);
                const T w = vr * rinvT;
                const T vsig = ci + cj - T(3) * w;
                const T rinv = T(2) / (rhoi + rhoj);
                pij = -T(0.5) * bal * alpha * vsig * w * rinv;
            }
            // artificial conductivity (src/fluid_force.cpp:108-116)
            T dac = 0;
            if(P.use_ac) {
                const T vs = P.gravity ? fabs(vr * rinvT) : sqrt(T(2) * fabs(Pi - Pj) / (rhoi + rhoj));
                dac = (T)P.alpha_ac * mj * vs * (ui - uj) * (dwij.x * rv.x + dwij.y * rv.y + dwij.z * rv.z) * rinvT;
            }
            const T vdwi = vij.x * dwi.x + vij.y * dwi.y + vij.z * dwi.z;
            const T vdwij = vij.x * dwij.x + vij.y * dwij.y + vij.z * dwij.z;
            T a_i, a_j, e_;
            if(TYPE == SPHGPU_DISPH || TYPE == SPHGPU_GDISPH) {
                const T fij = T(1) - (T)si.z / (mj * uj);
                const T fji = T(1) - (T)sj.z * mu_inv;
                a_i = mj * (g2up * uj * fij * psi + T(0.5) * pij);
                a_j = mj * (g2u * (uj / Pj) * fji * psj + T(0.5) * pij);
                e_ = mj * g2up * uj * fij * psi * vdwi + T(0.5) * mj * pij * vdwij + dac;
            } else {
                a_i = mj * (ppr * (T)si.z + T(0.5) * pij);
                a_j = mj * (Pj / (rhoj * rhoj) * (T)sj.z + T(0.5) * pij);
                e_ = mj * ppr * (T)si.z * vdwi + T(0.5) * mj * pij * vdwij + dac;
            }
            const T fx = dwi.x * a_i + dwj.x * a_j, fy = dwi.y * a_i + dwj.y * a_j, fz = dwi.z * a_i + dwj.z * a_j;
            ax -= (double)fx;
            ay -= (double)fy;
            az -= (double)fz;
            de += (double)e_;
            if constexpr(f32) sabs += fabsf(fx) + fabsf(fy) + fabsf(fz);
        }
        ax = group_sum<G>(ax);
        ay = group_sum<G>(ay);
        az = group_sum<G>(az);
        de = group_sum<G>(de);
        if constexpr(f32) sabs = group_sum<G>(sabs);
        if(MODE == 4) {
            if(cnt > 0 && lane == 0) {
                const double4 a0 = S.acc[i];
                S.acc[i] = make_double4(a0.x + ax, a0.y + ay, a0.z + az, a0.w + de);
                if(f32 && accabs) accabs[i] += sabs;
            }
        } else if(valid && lane == 0) {
            S.acc[i] = make_double4(ax, ay, az, de);
            if(f32 && accabs) accabs[i] = sabs;
        }
    }
    if(!sub.count) return;
    if(MODE != 4) {  // the completion pass re-solves pairs the force pass counted
        block_count(&st->force_cand, n_cand);
        block_count(&st->force_pairs, n_pairs);
    }
    if(TYPE == SPHGPU_GSPH) {
        for(int o = 16; o > 0; o >>= 1) {
            solves += __shfl_xor_sync(FULL_MASK, solves, o);
            iters += __shfl_xor_sync(FULL_MASK, iters, o);
            fallbacks += __shfl_xor_sync(FULL_MASK, fallbacks, o);
        }
        if((threadIdx.x & 31) == 0 && solves) {
            atomicAdd(&st->riemann_solves, solves);
            atomicAdd(&st->riemann_iters, iters);
            if(fallbacks) atomicAdd(&st->riemann_fallbacks, fallbacks);
        }
    }
}

constexpr int GROUP = 4;

unsigned force_grid(int n)
{
    const long long gpb = FBLK / GROUP;
    const long long blocks = (n + gpb - 1) / gpb;
    return (unsigned)std::max<long long>(1, std::min<long long>(blocks, 148LL * 8 * 4));
}

template <typename T, int MODE>
void launch_force(sphgpu_ctx* c, MlpPairs mp, Harvest hv, Subset sub = {nullptr, 0, 1})
{
    const unsigned grid = force_grid(sub.idx ? sub.n : c->n);
    const int type = c->prm.sph_type;
    float* accabs = sizeof(T) == sizeof(float) ? c->d_accabs : nullptr;
    if(type == SPHGPU_DISPH) {
        k_force<T, GROUP, SPHGPU_DISPH, 0><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist, c->d_pcount,
                                                                         (int)c->pcap, c->d_dt, c->d_status, mp, hv,
                                                                         accabs, sub);
    } else if(type == SPHGPU_GSPH) {
        k_force<T, GROUP, SPHGPU_GSPH, MODE><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist,
                                                                           c->d_pcount, (int)c->pcap, c->d_dt,
                                                                           c->d_status, mp, hv, accabs, sub);
    } else if(type == SPHGPU_GDISPH) {
        k_force<T, GROUP, SPHGPU_GDISPH, 0><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist,
                                                                          c->d_pcount, (int)c->pcap, c->d_dt,
                                                                          c->d_status, mp, hv, accabs, sub);
    } else {
        k_force<T, GROUP, SPHGPU_SSPH, 0><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist, c->d_pcount,
                                                                        (int)c->pcap, c->d_dt, c->d_status, mp, hv,
                                                                        accabs, sub);
    }
}

// Riemann problems in bulk (labels and evaluation of the learned guess).
// states: n x 7 (u_L, rho_L, p_L, u_R, rho_R, p_R, gamma).
__global__ void k_riemann_batch(const double* __restrict__ st, long long n, int mode, const float* __restrict__ y,
                                int budget, double* __restrict__ pstar, double* __restrict__ vstar,
                                int* __restrict__ iters, int* __restrict__ fb)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= n) return;
    const double* s = st + 7 * r;
    const double gamma = s[6];
    const double L[4] = {s[0], s[1], s[2], sqrt(gamma * s[2] / s[1])};
    const double R[4] = {s[3], s[4], s[5], sqrt(gamma * s[5] / s[4])};
    double p = 0.0, v = 0.0;
    int it = 0, f = 0;
    if(mode == 0) {
        riemann_iterative<double>(L, R, gamma, false, 0.f, budget, p, v, it, f);
    } else if(mode == 1) {
        riemann_iterative<double>(L, R, gamma, true, y[r], budget, p, v, it, f);
    } else {
        // plain start, Newton to a relative change of 1e-13 (mode 2, labels)
        // or 1e-10 (mode 3, the learned path's target accuracy)
        const double tol = mode == 2 ? 1e-13 : 1e-10;
        const double g2 = 1.0 + gamma, g1 = 0.5 * g2 / gamma;
        const double cl = sqrt(gamma * L[2] * L[1]), cr = sqrt(gamma * R[2] * R[1]);
        double q = R[2] - L[2] - cr * (R[0] - L[0]);
        q = fmax(L[2] + q * cl / (cl + cr), 1e-25);
        for(int k = 0; k < 100; ++k) {
            const double qo = q;
            q = vl_newton_step<double>(q, L[0], L[2], 1.0 / L[1], cl, R[0], R[2], 1.0 / R[1], cr, g1, g2);
            ++it;
            if(fabs(q - qo) / q < tol) break;
        }
        p = q;
        v = vl_ustar(q, L[0], L[2], cl, R[0], R[2], cr, g1);
    }
    pstar[r] = p;
    if(vstar) vstar[r] = v;
    if(iters) iters[r] = it;
    if(fb) fb[r] = f;
}

// One allocation for the deferred rows of the learned path (256-byte aligned
// pieces); with base == nullptr only the total size is computed.
struct DeferLayout {
    uint4* feat;
    uint64_t *keys, *keys_alt;
    float* y;
    uint32_t *vals, *vals_alt;
    void* scratch;
    int *dstart, *dcount;
    unsigned long long* rows;
    size_t total;
};

DeferLayout defer_layout(int64_t rcap, int64_t n, void* base)
{
    DeferLayout L{};
    char* b = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        void* p = b ? b + off : nullptr;
        off += (bytes + 255) & ~(size_t)255;
        return p;
    };
    L.feat = static_cast<uint4*>(take(sizeof(uint4) * (size_t)rcap));
    L.keys = static_cast<uint64_t*>(take(sizeof(uint64_t) * (size_t)rcap));
    L.keys_alt = static_cast<uint64_t*>(take(sizeof(uint64_t) * (size_t)rcap));
    L.y = static_cast<float*>(take(sizeof(float) * (size_t)rcap));
    L.vals = static_cast<uint32_t*>(take(sizeof(uint32_t) * (size_t)rcap));
    L.vals_alt = static_cast<uint32_t*>(take(sizeof(uint32_t) * (size_t)rcap));
    L.scratch = take(radix_scratch_bytes((int)rcap));
    L.dstart = static_cast<int*>(take(sizeof(int) * (size_t)n));
    L.dcount = static_cast<int*>(take(sizeof(int) * (size_t)n));
    L.rows = static_cast<unsigned long long*>(take(sizeof(unsigned long long)));
    L.total = off;
    return L;
}

__global__ void k_iota(uint32_t* v, int n)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if(r < n) v[r] = (uint32_t)r;
}

// Per particle, the first sorted row and the number of rows of its deferred pairs.
__global__ void k_defer_ranges(const uint64_t* __restrict__ skeys, int n, uint64_t cap, int* __restrict__ dstart,
                               int* __restrict__ dcount)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= n) return;
    const uint64_t p = skeys[r] / cap;
    if(r == 0 || skeys[r - 1] / cap != p) dstart[p] = r;
    atomicAdd(&dcount[p], 1);
}

}  // namespace

int fluid_force_subset64(sphgpu_ctx* c, const int* idx, int nsub)
{
    Harvest hv{};
    MlpPairs mp{};
    launch_force<double, 0>(c, mp, hv, Subset{idx, nsub, 0});
    SPHGPU_LAUNCH_CHECK(c, "FluidForce (FP64 re-evaluation)");
    return SPHGPU_OK;
}

int fluid_force(sphgpu_ctx* c)
{
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "FluidForce before tree make");
    if(c->prm.sph_type == SPHGPU_SRGSPH) return sr_fluid_force(c);
    const bool learned = c->prm.riemann_guess == SPHGPU_GUESS_MLP && c->prm.sph_type == SPHGPU_GSPH &&
                         c->prm.riemann_solver == SPHGPU_RIEMANN_ITERATIVE;
    if(learned && !c->have_mlp) return fail(c, SPHGPU_ERR_NO_MLP, "learned Riemann guess requested without MLP weights");
    const int rc_walk = symmetric_lists(c);
    if(rc_walk < 0) return rc_walk;
    {
        const int rc = ensure_recheck(c);
        if(rc < 0) return rc;
    }
    stage_begin(c, SPHGPU_T_FORCE);
    Harvest hv{c->d_harvest, c->d_harvest_count, c->harvest_cap, c->harvest_mod, 0u};
    MlpPairs mp{};
    int launches = 1;
    if(learned) {
        const int64_t slots = (int64_t)c->n * c->pcap;
        if(slots > 0xFFFFFFFFLL) return fail(c, SPHGPU_ERR_ARG, "learned guess: more than 2^32 pair slots");
        // room for 1/16 of all pair slots (the screen rejects well under 1%)
        // room for 1/16 of all pair slots, or for 1.25x the rows the last call
        // asked for (many strong shocks), at most one row per slot
        const int64_t rcap = std::min<int64_t>(
            std::max<int64_t>(std::max<int64_t>(1 << 20, slots / 16), c->mlp_rows_demand + c->mlp_rows_demand / 4),
            std::max<int64_t>(slots, 1 << 20));
        if(rcap > c->mlp_rcap || c->n > c->mlp_ncap) {
            if(c->d_mlp_defer) cudaFree(c->d_mlp_defer);
            c->d_mlp_defer = nullptr;
            c->mlp_rcap = 0;
            const size_t bytes = defer_layout(rcap, c->n, nullptr).total;
            SPHGPU_CUDA(c, cudaMalloc(&c->d_mlp_defer, bytes));
            c->mlp_rcap = rcap;
            c->mlp_ncap = c->n;
        }
        DeferLayout L = defer_layout(c->mlp_rcap, c->mlp_ncap, c->d_mlp_defer);
        SPHGPU_CUDA(c, cudaMemsetAsync(L.rows, 0, sizeof(unsigned long long), c->stream));
        mp.feat = L.feat;
        mp.keys = L.keys;
        mp.rows = L.rows;
        mp.rcap = c->mlp_rcap;
        // pass 1: every pair the screen accepts; the others become rows
        if(c->prm.precision == SPHGPU_MIXED) launch_force<float, 3>(c, mp, hv);
        else launch_force<double, 3>(c, mp, hv);
        SPHGPU_LAUNCH_CHECK(c, "FluidForce");
        unsigned long long rows = 0;
        SPHGPU_CUDA(c, cudaMemcpyAsync(&rows, L.rows, sizeof(rows), cudaMemcpyDeviceToHost, c->stream));
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        c->mlp_rows_demand = (int64_t)rows;  // the next call sizes its rows by it
        rows = std::min<unsigned long long>(rows, (unsigned long long)c->mlp_rcap);
        if(rows > 0) {
            const int nr = (int)rows;
            const int rc = mlp_infer_rows(c, L.feat, L.y, nr);
            if(rc < 0) return rc;
            // rows sorted by pair key: each particle's deferred pairs in slot order
            k_iota<<<grid_for(nr, 256), 256, 0, c->stream>>>(L.vals, nr);
            int bits = 1;
            while(bits < 32 && (1ull << bits) < (unsigned long long)slots) ++bits;
            uint64_t *kk = L.keys, *ka = L.keys_alt;
            uint32_t *vv = L.vals, *va = L.vals_alt;
            launches += 2 + radix_sort(kk, vv, ka, va, nr, (bits + 7) / 8 * 8, L.scratch, c->stream);
            SPHGPU_CUDA(c, cudaMemsetAsync(L.dcount, 0, sizeof(int) * (size_t)c->n, c->stream));
            k_defer_ranges<<<grid_for(nr, 256), 256, 0, c->stream>>>(kk, nr, (uint64_t)c->pcap, L.dstart, L.dcount);
            mp.y = L.y;
            mp.skeys = kk;
            mp.svals = vv;
            mp.dstart = L.dstart;
            mp.dcount = L.dcount;
            // pass 2: the deferred pairs from the network's guess, added to acc
            if(c->prm.precision == SPHGPU_MIXED) launch_force<float, 4>(c, mp, hv);
            else launch_force<double, 4>(c, mp, hv);
            launches += 2;
        }
    } else {
        if(c->prm.precision == SPHGPU_MIXED) launch_force<float, 0>(c, mp, hv);
        else launch_force<double, 0>(c, mp, hv);
    }
    SPHGPU_LAUNCH_CHECK(c, "FluidForce");
    stage_end(c, SPHGPU_T_FORCE, launches);
    c->accabs_valid = c->prm.precision == SPHGPU_MIXED;
    return rc_walk;
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int sphgpu_riemann_batch(sphgpu_ctx* c, const double* states, int64_t n, int mode, double* pstar, double* vstar,
                         int32_t* iters, int32_t* fallbacks)
{
    if(!c || !states || !pstar || n <= 0 || mode < 0 || mode > 3) return SPHGPU_ERR_ARG;
    if(!c->stream) return fail(c, SPHGPU_ERR_CUDA, "context has no device");
    if(mode == 1 && !c->have_mlp) return fail(c, SPHGPU_ERR_NO_MLP, "no MLP parameters loaded");
    double *d_st = nullptr, *d_p = nullptr, *d_v = nullptr;
    int *d_it = nullptr, *d_fb = nullptr;
    float* d_y = nullptr;
    DevTemps tmp(c->stream);
    SPHGPU_CUDA(c, tmp.get(&d_st, sizeof(double) * 7 * (size_t)n, false));
    SPHGPU_CUDA(c, cudaMemcpyAsync(d_st, states, sizeof(double) * 7 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    SPHGPU_CUDA(c, tmp.get(&d_p, sizeof(double) * (size_t)n, false));
    SPHGPU_CUDA(c, tmp.get(&d_v, sizeof(double) * (size_t)n, false));
    SPHGPU_CUDA(c, tmp.get(&d_it, sizeof(int) * (size_t)n, false));
    SPHGPU_CUDA(c, tmp.get(&d_fb, sizeof(int) * (size_t)n, false));
    if(mode == 1) {
        SPHGPU_CUDA(c, tmp.get(&d_y, sizeof(float) * (size_t)n, false));
        const int rc = mlp_predict_states(c, d_st, n, d_y);
        if(rc < 0) return rc;
    }
    const int budget = mode == 1 ? c->prm.mlp_max_newton : 20;
    k_riemann_batch<<<grid_for(n, 256), 256, 0, c->stream>>>(d_st, n, mode, d_y, budget, d_p, d_v, d_it, d_fb);
    SPHGPU_LAUNCH_CHECK(c, "riemann batch");
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));  // the context stream does not sync with cudaMemcpy
    SPHGPU_CUDA(c, cudaMemcpy(pstar, d_p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
    if(vstar) SPHGPU_CUDA(c, cudaMemcpy(vstar, d_v, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
    if(iters) SPHGPU_CUDA(c, cudaMemcpy(iters, d_it, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    if(fallbacks) SPHGPU_CUDA(c, cudaMemcpy(fallbacks, d_fb, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    return SPHGPU_OK;
}

// Collect pair states from the plain solver: the next FluidForce calls
// append every pair with hash(i, k) % sample_mod == 0 (up to capacity
// records of 8 doubles).  sphgpu_harvest_end copies them out and stops.
int sphgpu_harvest_begin(sphgpu_ctx* c, int64_t capacity, uint32_t sample_mod)
{
    if(!c || capacity <= 0 || sample_mod == 0) return SPHGPU_ERR_ARG;
    if(c->d_harvest) cudaFree(c->d_harvest);
    if(c->d_harvest_count) cudaFree(c->d_harvest_count);
    SPHGPU_CUDA(c, cudaMalloc(&c->d_harvest, sizeof(double) * 8 * (size_t)capacity));
    SPHGPU_CUDA(c, cudaMalloc(&c->d_harvest_count, sizeof(unsigned long long)));
    SPHGPU_CUDA(c, cudaMemsetAsync(c->d_harvest_count, 0, sizeof(unsigned long long), c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    c->harvest_cap = capacity;
    c->harvest_mod = sample_mod;
    return SPHGPU_OK;
}

int sphgpu_harvest_end(sphgpu_ctx* c, double* out, int64_t capacity, int64_t* count)
{
    if(!c || !count) return SPHGPU_ERR_ARG;
    *count = 0;
    if(!c->d_harvest) return fail(c, SPHGPU_ERR_STATE, "no harvest in progress");
    unsigned long long n = 0;
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    SPHGPU_CUDA(c, cudaMemcpy(&n, c->d_harvest_count, sizeof(n), cudaMemcpyDeviceToHost));
    const int64_t m = std::min<int64_t>(std::min<int64_t>((int64_t)n, c->harvest_cap), capacity);
    if(out && m > 0) SPHGPU_CUDA(c, cudaMemcpy(out, c->d_harvest, sizeof(double) * 8 * (size_t)m, cudaMemcpyDeviceToHost));
    *count = m;
    cudaFree(c->d_harvest);
    cudaFree(c->d_harvest_count);
    c->d_harvest = nullptr;
    c->d_harvest_count = nullptr;
    c->harvest_cap = 0;
    c->harvest_mod = 0;
    return SPHGPU_OK;
}

}  // extern "C"
