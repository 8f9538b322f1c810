// force.cu — FluidForce::calculation for ssph, disph and gsph.
//
// Reference: src/fluid_force.cpp:26-116 (ssph pair force, Monaghan-97
// artificial viscosity, artificial conductivity), src/disph/d_fluid_force.cpp:26-86
// (Hopkins-2013 pressure-energy force), src/gsph/g_fluid_force.cpp:32-304
// (van Leer limiter, MUSCL reconstruction, HLL and iterative Riemann solvers).
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

// Iterative solver (src/gsph/g_fluid_force.cpp:209-304).  Plain form: FP64
// throughout.  Mixed form: iterations in T = float, then one FP64 Newton step
// and the FP64 u*.  With `guess` > 0 (learned form) Newton starts from the
// guess, runs at most `budget` iterations to a 1e-10 relative change (the
// last checked in FP64) and falls back to the plain start on failure.
template <typename T>
__device__ void riemann_iterative(const double* L, const double* R, double gamma, double guess, int budget,
                                  double& pstar, double& vstar, int& iters, int& fallback)
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
    if(guess > 0.0) {
        // learned start: Newton to 1e-10, FP32 iterations + FP64 check
        p = guess;
        bool ok = false;
        for(int it = 0; it < budget; ++it) {
            const double pold = p;
            p = vl_newton_step<double>(p, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
            ++iters;
            if(fabs(p - pold) / p < 1e-10) {
                ok = true;
                break;
            }
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
    if(sizeof(T) == sizeof(double)) {
        p = pg;
        for(int it = 0; it < 20; ++it) {
            const double pold = p;
            p = vl_newton_step<double>(p, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
            ++iters;
            if(fabs(p - pold) / p < 1e-6) break;
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
        // final Newton step in FP64
        p = vl_newton_step<double>((double)pf, ul, pl, vl, cl, ur, pr, vr, cr, g1, g2);
    }
    pstar = p;
    vstar = vl_ustar(p, ul, pl, cl, ur, pr, cr, g1);
}

template <typename T, int G, int TYPE>
__global__ void __launch_bounds__(FBLK) k_force(DevParams P, DevState S, int n, const int* __restrict__ list,
                                                const int* __restrict__ count, int cap, const double* __restrict__ dtp,
                                                DevStatus* __restrict__ st, MlpDev mlp)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * FBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * FBLK) >> 5;
    const double dt = *dtp;
    const double gamma = P.gamma;
    unsigned long long solves = 0, iters = 0, fallbacks = 0;

    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        const bool valid = i < n;
        const int cnt = valid ? min(count[i], cap) : 0;
        const int* li = list + (size_t)(valid ? i : 0) * (size_t)cap;
        const double4 pi = valid ? S.pos[i] : make_double4(0, 0, 0, 0);
        const double4 vi = valid ? S.vel[i] : make_double4(0, 0, 0, 1);
        const double4 ti = valid ? S.thermo[i] : make_double4(1, 1, 1, 1);
        const double4 si = valid ? S.visc[i] : make_double4(0, 0, 1, 0);
        const double hi = vi.w;
        double4 gi0 = make_double4(0, 0, 0, 0), gi1 = gi0, gi2 = gi0, gi3 = gi0;
        if(TYPE == SPHGPU_GSPH && P.gsph2 && valid) {
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
        for(int k = lane; k < cnt; k += G) {
            const int j = li[k];
            const double4 pj = S.pos[j];
            const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double r = sqrt(abs2x(d));
            const double4 vj = S.vel[j];
            const double hj = vj.w;
            if(r >= (hi < hj ? hj : hi) || r == 0.0) continue;
            const double4 tj = S.thermo[j];
            const T rT = (T)r;
            const T rinvT = (T)(1.0 / r);
            const V3<T> rv{(T)d.x, (T)d.y, (T)d.z};
            const KernH<T> khj(P.kernel, (T)hj);
            const T ci_ = khi.dwc(rT, rinvT);
            const T cj_ = khj.dwc(rT, rinvT);
            const V3<T> dwi{rv.x * ci_, rv.y * ci_, rv.z * ci_};
            const V3<T> dwj{rv.x * cj_, rv.y * cj_, rv.z * cj_};
            const T mj = (T)pj.w;
            const T rhoj = (T)tj.x, Pj = (T)tj.y, uj = (T)tj.z, cj = (T)tj.w;
            if(TYPE == SPHGPU_GSPH) {
                const double rinv = 1.0 / r;
                const double ex = d.x * rinv, ey = d.y * rinv, ez = d.z * rinv;
                const double vei = vi.x * ex + vi.y * ey + vi.z * ez;
                const double vej = vj.x * ex + vj.y * ey + vj.z * ez;
                double Lst[4], Rst[4];
                if(P.gsph2) {
                    // MUSCL reconstruction (src/gsph/g_fluid_force.cpp:103-140)
                    const double4 gj0 = S.grad[j], gj1 = S.grad[(size_t)n + j];
                    const double4 gj2 = S.grad[2 * (size_t)n + j], gj3 = S.grad[3 * (size_t)n + j];
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
                double pstar, vstar;
                if(P.riemann == SPHGPU_RIEMANN_ITERATIVE) {
                    double guess = -1.0;
                    if(mlp.w != nullptr) guess = mlp_guess(mlp, Lst, Rst, gamma);
                    int it = 0, fb = 0;
                    riemann_iterative<T>(Lst, Rst, gamma, guess, P.mlp_max_newton, pstar, vstar, it, fb);
                    ++solves;
                    iters += it;
                    fallbacks += fb;
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
                de -= fx * (ex * vstar - vi.x) + fy * (ey * vstar - vi.y) + fz * (ez * vstar - vi.z);
                continue;
            }
            const double4 sj = S.visc[j];
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
            if(TYPE == SPHGPU_DISPH) {
                const T fij = T(1) - (T)si.z / (mj * uj);
                const T fji = T(1) - (T)sj.z * mu_inv;
                a_i = mj * (g2up * uj * fij + T(0.5) * pij);
                a_j = mj * (g2u * (uj / Pj) * fji + T(0.5) * pij);
                e_ = mj * g2up * uj * fij * vdwi + T(0.5) * mj * pij * vdwij + dac;
            } else {
                a_i = mj * (ppr * (T)si.z + T(0.5) * pij);
                a_j = mj * (Pj / (rhoj * rhoj) * (T)sj.z + T(0.5) * pij);
                e_ = mj * ppr * (T)si.z * vdwi + T(0.5) * mj * pij * vdwij + dac;
            }
            ax -= (double)(dwi.x * a_i + dwj.x * a_j);
            ay -= (double)(dwi.y * a_i + dwj.y * a_j);
            az -= (double)(dwi.z * a_i + dwj.z * a_j);
            de += (double)e_;
        }
        ax = group_sum<G>(ax);
        ay = group_sum<G>(ay);
        az = group_sum<G>(az);
        de = group_sum<G>(de);
        if(valid && lane == 0) S.acc[i] = make_double4(ax, ay, az, de);
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

constexpr int GROUP = 8;

unsigned force_grid(int n)
{
    const long long gpb = FBLK / GROUP;
    const long long blocks = (n + gpb - 1) / gpb;
    return (unsigned)std::max<long long>(1, std::min<long long>(blocks, 148LL * 8 * 4));
}

template <typename T>
void launch_force(sphgpu_ctx* c, MlpDev m)
{
    const unsigned grid = force_grid(c->n);
    const int type = c->prm.sph_type;
    if(type == SPHGPU_DISPH) {
        k_force<T, GROUP, SPHGPU_DISPH><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist, c->d_pcount,
                                                                      (int)c->pcap, c->d_dt, c->d_status, m);
    } else if(type == SPHGPU_GSPH) {
        k_force<T, GROUP, SPHGPU_GSPH><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist, c->d_pcount,
                                                                     (int)c->pcap, c->d_dt, c->d_status, m);
    } else {
        k_force<T, GROUP, SPHGPU_SSPH><<<grid, FBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist, c->d_pcount,
                                                                     (int)c->pcap, c->d_dt, c->d_status, m);
    }
}

}  // namespace

int fluid_force(sphgpu_ctx* c)
{
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "FluidForce before tree make");
    MlpDev m{};
    if(c->prm.riemann_guess == SPHGPU_GUESS_MLP && c->prm.sph_type == SPHGPU_GSPH) {
        if(!c->have_mlp) return fail(c, SPHGPU_ERR_NO_MLP, "learned Riemann guess requested without MLP weights");
        m = mlp_device(c);
    }
    const int rc_walk = pair_walk(c);
    if(rc_walk < 0) return rc_walk;
    stage_begin(c, SPHGPU_T_FORCE);
    if(c->prm.precision == SPHGPU_MIXED) launch_force<float>(c, m);
    else launch_force<double>(c, m);
    SPHGPU_LAUNCH_CHECK(c, "FluidForce");
    stage_end(c, SPHGPU_T_FORCE, 1);
    return rc_walk;
}

}  // namespace sphgpu
