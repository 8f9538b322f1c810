// srgsph.cu — special-relativistic Godunov SPH (SRGSPH): PreInteraction,
// FluidForce, TimeStep and the conserved-variable kick-drift.
//
// Reference: src/srgsph/sr_pre_interaction.cpp:31-407,
// src/srgsph/sr_fluid_force.cpp:47-480, src/srgsph/sr_primitive_recovery.cpp:23-160,
// src/srgsph/sr_timestep.cpp:14-59, and the SRGSPH branches of Solver::predict /
// correct (src/solver.cpp:992-1043, 1075-1102); Kitajima, Inutsuka & Seno (2025).
//
// State per particle (DevState::sr, 4 x n double4): {S, e} conserved momentum
// and energy, {N, nu, gamma_lor, H} lab-frame baryon density, baryons per
// particle, Lorentz factor and specific enthalpy, {dS/dt, de/dt}, {N before
// the current pre-interaction}.  The primitives (v, n = N / gamma_lor, P, c_s)
// follow from PrimitiveRecovery: gamma_lor, v and H depend on (S, e) only, n
// and P also on N.
//
// Layout of the work: G = 4 lanes per particle over the ELL lists (gather list
// for the pre-interaction, symmetric list for the force), group-reduced sums.
// FP64 throughout, unfused (-fmad=false for this file), so the primitive
// recovery and the kick-drift are bit-identical to the reference's on the
// same inputs; the list sums run in a different order than the reference's
// distance-sorted lists, and pow / log10 are CUDA's, so the pre-interaction
// and force agree with the reference to rounding.
//
// The reference's pre-interaction loop updates N_i while the same loop reads
// the neighbours' N for their volumes and primitives, so its result depends on
// the loop order; single-threaded, particle j < i has its new N and j > i its
// old one when i is processed.  The gradient pass here keeps both and selects
// by the caller index (DevState::id), reproducing that order on the GPU.
#include <algorithm>
#include <cfloat>
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int SBLK = 128;
constexpr int SG = 4;  // lanes per particle

// PrimitiveRecovery::solve_lorentz_factor: Newton on
// (g^2 - 1)(X e g - 1)^2 - S^2 (X g^2 - 1)^2 / c^2 = 0, X = G / (G - 1),
// at most 100 iterations to a 1e-10 relative step.
__device__ bool sr_lorentz(double S_mag, double e, double ge, double c, double& g)
{
    const double X = ge / (ge - 1.0);
    const double c2 = c * c;
    const double S2 = S_mag * S_mag;
    g = 1.0 + sqrt(1.0 + S2 / c2) / X;
    for(int it = 0; it < 100; ++it) {
        const double g2 = g * g;
        const double g2m1 = g2 - 1.0;
        const double xe = X * e * g - 1.0;
        const double xg = X * g2 - 1.0;
        const double f = g2m1 * xe * xe - S2 * xg * xg / c2;
        const double df = 2.0 * g * xe * xe + 2.0 * g2m1 * xe * X * e - 2.0 * S2 * xg * 2.0 * X * g / c2;
        const double delta = f / df;
        g -= delta;
        if(g < 1.0) g = 1.0 + 1.0e-10;
        if(fabs(delta) < 1.0e-10 * g) return true;
    }
    return false;
}

// The N-independent part of conserved_to_primitive: gamma_lor, v, H.
struct SRKin {
    double vx, vy, vz, g, H;
};

__device__ bool sr_kin(double Sx, double Sy, double Sz, double e, double ge, double c, SRKin& k)
{
    const double S_mag = sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
    if(!sr_lorentz(S_mag, e, ge, c, k.g)) return false;
    const double X = ge / (ge - 1.0);
    const double g = k.g, g2 = g * g;
    const double num = X * g2 - 1.0;
    const double den = g * (X * e * g - 1.0);
    const double f = num / den;
    k.vx = Sx * f;
    k.vy = Sy * f;
    k.vz = Sz * f;
    const double v_mag = sqrt(k.vx * k.vx + k.vy * k.vy + k.vz * k.vz);
    const double c2 = c * c;
    k.H = v_mag > 1.0e-10 ? S_mag / (g * v_mag) : 1.0 + (e - 1.0) / c2;
    return true;
}

// rest-frame density and pressure at lab-frame density N
__device__ __forceinline__ void sr_eos(double g, double H, double N, double ge, double c, double& dens,
                                       double& pres)
{
    dens = N / g;
    pres = (ge - 1.0) * dens * (c * c) * (H - 1.0) / ge;
}

__device__ __forceinline__ double sr_sound(double H, double ge) { return sqrt((ge - 1.0) * (H - 1.0) / H); }

__device__ __forceinline__ double wrap(const DevParams& P, double x, int k)
{
    if(!P.periodic) return x;
    if(x < P.lo[k]) return x + P.range[k];
    if(x > P.hi[k]) return x - P.range[k];
    return x;
}

// ------------------------------------------------------------ pre-interaction
// initial_smoothing: h = eta (nu / N)^(1/3)
__global__ void k_sr_initial_sml(DevParams P, DevState S, int n)
{
    const int i = blockIdx.x * SBLK + threadIdx.x;
    if(i >= n) return;
    const double4 aux = S.sr[(size_t)n + i];
    S.vel[i].w = P.sr_eta * pow(aux.y / aux.x, 1.0 / 3);
}

// gamma_lor, v, H of every particle from (S, e)
__global__ void k_sr_kin(DevParams P, DevState S, int n, DevStatus* __restrict__ st)
{
    const int i = blockIdx.x * SBLK + threadIdx.x;
    if(i >= n) return;
    const double4 se = S.sr[i];
    SRKin k;
    if(!sr_kin(se.x, se.y, se.z, se.w, P.gamma, P.sr_c, k)) {
        st->sr_recovery = 1;
        return;
    }
    double4 v = S.vel[i];
    v.x = k.vx;
    v.y = k.vy;
    v.z = k.vz;
    S.vel[i] = v;
    double4& aux = S.sr[(size_t)n + i];
    aux.z = k.g;
    aux.w = k.H;
}

// Smoothing length (compute_smoothing_length: damped fixed point
// h <- (h + eta Vp*^(1/3)) / 2 with Vp* = 1 / sum W(r, C_smooth h), or the
// non-iterative h = eta (nu / N)^(1/3)), then the volume Vp = 1 / sum W(r, h)
// (compute_volume) and N = nu / Vp.  Both sums run over the gather list
// (self included) plus one more self term, as the reference's do.
template <int G>
__global__ void __launch_bounds__(SBLK) k_sr_pre_h(DevParams P, DevState S, int n, const int* __restrict__ list,
                                                   const int* __restrict__ count, int cap)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * SBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * SBLK) >> 5;
    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        if(i >= n) continue;  // whole groups drop out together
        const int cnt = min(count[i], cap);
        const int* li = list + (size_t)i * (size_t)cap;
        const double4 pi = S.pos[i];
        const double4 aux = S.sr[(size_t)n + i];
        const double nu = aux.y, Nold = aux.x;
        double h = S.vel[i].w;
        if(P.iterative) {
            for(int iter = 0; iter < 20; ++iter) {
                const double hs = P.sr_c_smooth * h;
                const KernH<double> kh(P.kernel, hs);
                double sum = 0.0;
                for(int k = lane; k < cnt; k += G) {
                    const double4 pj = S.pos[li[k]];
                    const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
                    const double r = sqrt(abs2x(d));
                    if(r < hs) sum += kh.w(r);
                }
                sum = group_sum<G>(sum) + kh.w(0.0);
                if(sum < 1.0e-20) {
                    h *= 1.5;
                    continue;
                }
                const double hn = P.sr_eta * pow(1.0 / sum, 1.0 / 3.0);
                const double hd = 0.5 * (h + hn);
                if(fabs(hd - h) < 1.0e-6 * h) {
                    h = hd;
                    break;
                }
                h = hd;
                if(h < 1.0e-10) h = 1.0e-10;
                if(h > 10.0) h = 10.0;
            }
        } else {
            h = P.sr_eta * pow(nu / Nold, 1.0 / 3);
        }
        const KernH<double> kh(P.kernel, h);
        double sw = 0.0;
        for(int k = lane; k < cnt; k += G) {
            const double4 pj = S.pos[li[k]];
            const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double r = sqrt(abs2x(d));
            if(r < h) sw += kh.w(r);
        }
        sw = group_sum<G>(sw) + kh.w(0.0);
        if(lane == 0) {
            S.vel[i].w = h;
            S.sr[3 * (size_t)n + i].x = Nold;
            S.sr[(size_t)n + i].x = nu / (1.0 / sw);
        }
    }
}

// Primitives of i at its new N, and the MUSCL gradients
// grad q_i = sum_j V_j (q_j - q_i) grad W(r, h_i) / sum_j V_j W(r, h_i),
// V_j = nu_j / N_j, q = n, P, v (src/srgsph/sr_pre_interaction.cpp:336-405).
template <int G>
__global__ void __launch_bounds__(SBLK) k_sr_pre_grad(DevParams P, DevState S, int n, const int* __restrict__ list,
                                                      const int* __restrict__ count, int cap)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * SBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * SBLK) >> 5;
    const double ge = P.gamma, c = P.sr_c;
    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        if(i >= n) continue;
        const int cnt = min(count[i], cap);
        const int* li = list + (size_t)i * (size_t)cap;
        const double4 pi = S.pos[i];
        const double4 vi = S.vel[i];
        const double4 aux = S.sr[(size_t)n + i];
        const double h = vi.w;
        double dens_i, pres_i;
        sr_eos(aux.z, aux.w, aux.x, ge, c, dens_i, pres_i);
        const int idi = S.id[i];
        const KernH<double> kh(P.kernel, h);
        double om = 0.0, a[15];
#pragma unroll
        for(int q = 0; q < 15; ++q) a[q] = 0.0;
        for(int k = lane; k < cnt; k += G) {
            const int j = li[k];
            const double4 pj = S.pos[j];
            const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double r = sqrt(abs2x(d));
            if(r >= h || r == 0.0) continue;
            const double4 auxj = S.sr[(size_t)n + j];
            // N of j as the reference's serial loop sees it when it reaches i
            const double Nj = S.id[j] < idi ? auxj.x : S.sr[3 * (size_t)n + j].x;
            double dens_j, pres_j;
            sr_eos(auxj.z, auxj.w, Nj, ge, c, dens_j, pres_j);
            const double4 vj = S.vel[j];
            const double cw = kh.dwc(r, 1.0 / r);
            const double dwx = d.x * cw, dwy = d.y * cw, dwz = d.z * cw;
            const double vol = auxj.y / Nj;
            om += vol * kh.w(r);
            const double q[5] = {vol * (dens_j - dens_i), vol * (pres_j - pres_i), vol * (vj.x - vi.x),
                                 vol * (vj.y - vi.y), vol * (vj.z - vi.z)};
#pragma unroll
            for(int g = 0; g < 5; ++g) {
                a[3 * g] += dwx * q[g];
                a[3 * g + 1] += dwy * q[g];
                a[3 * g + 2] += dwz * q[g];
            }
        }
        om = group_sum<G>(om);
#pragma unroll
        for(int q = 0; q < 15; ++q) a[q] = group_sum<G>(a[q]);
        if(lane == 0) {
            const double oi = om > 0.0 ? 1.0 / om : 0.0;
            double b[16];
#pragma unroll
            for(int q = 0; q < 15; ++q) b[q] = om > 0.0 ? a[q] * oi : 0.0;
            b[15] = 0.0;
#pragma unroll
            for(int g = 0; g < 4; ++g)
                S.grad[(size_t)g * n + i] = make_double4(b[4 * g], b[4 * g + 1], b[4 * g + 2], b[4 * g + 3]);
            double4 t = S.thermo[i];
            t.x = dens_i;
            t.y = pres_i;
            t.w = sr_sound(aux.w, ge);
            S.thermo[i] = t;
        }
    }
}

// ------------------------------------------------------------ Riemann solver
// Exact SR Riemann solver of FluidForce::exact_riemann_solver
// (src/srgsph/sr_fluid_force.cpp:236-350; Pons, Marti & Mueller 2000), with
// its shock branch (Taub adiabat, :366-420) and its rarefaction branch (100
// explicit Euler steps along the isentrope, :436-480).  Normal velocities
// only; damped Newton with a numerical derivative, at most 50 iterations.
__device__ double sr_shock_velocity(double ge, double p_a, double rho_a, double h_a, double vx_a, double W_a,
                                    double p_b, bool left)
{
    const double dp = p_a - p_b;
    const double A = 1.0 + (ge - 1.0) * dp / (ge * p_b);
    const double B = -h_a * dp / (ge * p_b);
    const double Cc = -h_a * h_a + h_a * dp / rho_a;
    const double disc = B * B - 4.0 * A * Cc;
    if(disc < 0.0) return vx_a;
    const double h_b = (-B + sqrt(disc)) / (2.0 * A);
    const double rho_b = ge * p_b / ((ge - 1.0) * (h_b - 1.0));
    const double hra = h_a / rho_a;
    const double hrb = h_b / rho_b;
    const double j2 = -(p_b - p_a) / (hrb - hra);
    if(j2 < 0.0) return vx_a;
    const double j = left ? -sqrt(j2) : sqrt(j2);
    const double rwa = rho_a * W_a;
    const double rwa2 = rwa * rwa;
    const double numer = rwa2 * vx_a + j * sqrt(j2 + rwa2 * (1.0 - vx_a * vx_a));
    const double denom = rwa2 + j2;
    const double Vs = numer / denom;
    const double Ws = 1.0 / sqrt(1.0 - Vs * Vs);
    const double t1 = h_a * W_a * vx_a + Ws * (p_b - p_a) / j + Ws * Vs / (rho_a * W_a);
    const double t2 = h_a * W_a + (p_b - p_a) / j;
    return t2 / t1;
}

__device__ double sr_rarefaction_velocity(double ge, double p_a, double rho_a, double vx_a, double p_b, bool left)
{
    const double dp = (p_b - p_a) / 100;
    double p = p_a, vx = vx_a;
    const double sign = left ? -1.0 : 1.0;
    for(int k = 0; k < 100; ++k) {
        const double eps = (ge - 1.0) * p / rho_a;
        const double rho = rho_a * pow(p / p_a, 1.0 / ge);
        const double h = 1.0 + eps + p / rho;
        const double cs = sqrt(ge * p / (rho * h));
        const double W = 1.0 / sqrt(1.0 - vx * vx);
        const double dvdp = sign / (rho * h * W * W * cs);
        vx += dvdp * dp;
        p += dp;
        if(vx >= 1.0) vx = 0.99999;
        if(vx <= -1.0) vx = -0.99999;
    }
    return vx;
}

__device__ __forceinline__ double sr_wave(double ge, double ps, double p_a, double rho_a, double h_a, double vx_a,
                                          double W_a, bool left)
{
    return ps > p_a ? sr_shock_velocity(ge, p_a, rho_a, h_a, vx_a, W_a, ps, left)
                    : sr_rarefaction_velocity(ge, p_a, rho_a, vx_a, ps, left);
}

// state = (v, n, P, c_s)
__device__ __noinline__ void sr_riemann(double ge, const double* L, const double* R, double& pstar, double& vstar)
{
    const double vL = L[0], nL = L[1], pL = L[2];
    const double vR = R[0], nR = R[1], pR = R[2];
    const double hL = 1.0 + ge * pL / ((ge - 1.0) * nL);
    const double hR = 1.0 + ge * pR / ((ge - 1.0) * nR);
    const double WL = 1.0 / sqrt(1.0 - vL * vL);
    const double WR = 1.0 / sqrt(1.0 - vR * vR);
    double ps = 0.5 * (pL + pR);
    for(int it = 0; it < 50; ++it) {
        const double vLs = sr_wave(ge, ps, pL, nL, hL, vL, WL, true);
        const double vRs = sr_wave(ge, ps, pR, nR, hR, vR, WR, false);
        const double f = vRs - vLs;
        if(fabs(f) < 1.0e-8) {
            pstar = ps;
            vstar = 0.5 * (vLs + vRs);
            return;
        }
        const double dp = ps * 1.0e-6;
        const double vLp = sr_wave(ge, ps + dp, pL, nL, hL, vL, WL, true);
        const double vRp = sr_wave(ge, ps + dp, pR, nR, hR, vR, WR, false);
        const double fp = vRp - vLp;
        const double df = (fp - f) / dp;
        if(fabs(df) > 1.0e-12) {
            double pn = ps - 0.5 * f / df;
            pn = fmax(pn, 0.01 * fmin(pL, pR));
            ps = pn;
        } else if(f > 0) {
            ps *= 0.9;
        } else {
            ps *= 1.1;
        }
    }
    const double vLs = sr_wave(ge, ps, pL, nL, hL, vL, WL, true);
    const double vRs = sr_wave(ge, ps, pR, nR, hR, vR, WR, false);
    pstar = ps;
    vstar = 0.5 * (vLs + vRs);
}

__device__ __forceinline__ double limiter(double dq1, double dq2)
{
    const double p = dq1 * dq2;
    return p <= 0 ? 0.0 : 2.0 * p / (dq1 + dq2);
}

// ------------------------------------------------------------ force
// nu_i dS_i/dt = -sum_j P* V2_ij (grad W(r, 2 h_i) - grad W(r, 2 h_j)),
// nu_i de_i/dt = -sum_j P* v* e_ij . V2_ij (...), V2_ij = (V_i^2 + V_j^2) / 2
// over pairs with r < max(h_i, h_j) (src/srgsph/sr_fluid_force.cpp:47-232).
template <int G>
__global__ void __launch_bounds__(SBLK) k_sr_force(DevParams P, DevState S, int n, const int* __restrict__ list,
                                                   const int* __restrict__ count, int cap,
                                                   const double* __restrict__ dtp)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * SBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * SBLK) >> 5;
    const double ge = P.gamma, dt = *dtp;
    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        if(i >= n) continue;
        const int cnt = min(count[i], cap);
        const int* li = list + (size_t)i * (size_t)cap;
        const double4 pi = S.pos[i], vi = S.vel[i], ti = S.thermo[i];
        const double4 auxi = S.sr[(size_t)n + i];
        const double hi = vi.w, ci = ti.w, Pi = ti.y, Ni = auxi.x, nui = auxi.y, gi = auxi.z;
        double4 gi0 = make_double4(0, 0, 0, 0), gi1 = gi0, gi2 = gi0, gi3 = gi0;
        if(P.sr_2nd) {
            gi0 = S.grad[i];
            gi1 = S.grad[(size_t)n + i];
            gi2 = S.grad[2 * (size_t)n + i];
            gi3 = S.grad[3 * (size_t)n + i];
        }
        const KernH<double> khi(P.kernel, 2.0 * hi);
        double sx = 0.0, sy = 0.0, sz = 0.0, de = 0.0;
        for(int k = lane; k < cnt; k += G) {
            const int j = li[k];
            const double4 pj = S.pos[j], vj = S.vel[j];
            const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double r = sqrt(abs2x(d));
            const double hj = vj.w;
            if(r >= fmax(hi, hj) || r == 0.0) continue;
            const double4 tj = S.thermo[j];
            const double4 auxj = S.sr[(size_t)n + j];
            const double cj = tj.w, Pj = tj.y, Nj = auxj.x, gj = auxj.z;
            const double rinv = 1.0 / r;
            const double ex = d.x * rinv, ey = d.y * rinv, ez = d.z * rinv;
            const double vei = vi.x * ex + vi.y * ey + vi.z * ez;
            const double vej = vj.x * ex + vj.y * ey + vj.z * ez;
            const double n_i = Ni / gi, n_j = Nj / gj;
            double right[4] = {vei, n_i, Pi, ci}, left[4] = {vej, n_j, Pj, cj};
            if(P.sr_2nd) {
                const double min_cs = fmin(ci, cj);
                const double shock = P.sr_c_shock * fabs(vei - vej);
                const double pjump = fabs(log10(Pi / Pj));
                if(!((shock > min_cs) || (pjump > P.sr_c_cd))) {
                    const double4 gj0 = S.grad[j], gj1 = S.grad[(size_t)n + j];
                    const double4 gj2 = S.grad[2 * (size_t)n + j], gj3 = S.grad[3 * (size_t)n + j];
                    const double di = 0.5 * (1.0 - ci * dt * rinv);
                    const double dj = 0.5 * (1.0 - cj * dt * rinv);
                    const double dv = vei - vej;
                    const double dvi0 = gi1.z * ex + gi1.w * ey + gi2.x * ez;
                    const double dvi1 = gi2.y * ex + gi2.z * ey + gi2.w * ez;
                    const double dvi2 = gi3.x * ex + gi3.y * ey + gi3.z * ez;
                    const double dvj0 = gj1.z * ex + gj1.w * ey + gj2.x * ez;
                    const double dvj1 = gj2.y * ex + gj2.z * ey + gj2.w * ez;
                    const double dvj2 = gj3.x * ex + gj3.y * ey + gj3.z * ez;
                    const double dve_i = (dvi0 * ex + dvi1 * ey + dvi2 * ez) * r;
                    const double dve_j = (dvj0 * ex + dvj1 * ey + dvj2 * ez) * r;
                    right[0] = vei - limiter(dv, dve_i) * di;
                    left[0] = vej + limiter(dv, dve_j) * dj;
                    const double dn = n_i - n_j;
                    const double dn_i = (gi0.x * ex + gi0.y * ey + gi0.z * ez) * r / gi;
                    const double dn_j = (gj0.x * ex + gj0.y * ey + gj0.z * ez) * r / gj;
                    right[1] = n_i - limiter(dn, dn_i) * di;
                    left[1] = n_j + limiter(dn, dn_j) * dj;
                    const double dpp = Pi - Pj;
                    const double dp_i = (gi0.w * ex + gi1.x * ey + gi1.y * ez) * r;
                    const double dp_j = (gj0.w * ex + gj1.x * ey + gj1.y * ez) * r;
                    right[2] = Pi - limiter(dpp, dp_i) * di;
                    left[2] = Pj + limiter(dpp, dp_j) * dj;
                    right[3] = sqrt(ge * right[2] / right[1]);
                    left[3] = sqrt(ge * left[2] / left[1]);
                }
            }
            double pstar, vstar;
            sr_riemann(ge, left, right, pstar, vstar);
            const KernH<double> khj(P.kernel, 2.0 * hj);
            const double ci_ = khi.dwc(r, rinv), cj_ = khj.dwc(r, rinv);
            const double wx = d.x * ci_ - d.x * cj_;
            const double wy = d.y * ci_ - d.y * cj_;
            const double wz = d.z * ci_ - d.z * cj_;
            const double Vi = nui / Ni, Vj = auxj.y / Nj;
            const double pv = pstar * (0.5 * (Vi * Vi + Vj * Vj));
            sx -= wx * pv;
            sy -= wy * pv;
            sz -= wz * pv;
            de -= ((ex * vstar) * wx + (ey * vstar) * wy + (ez * vstar) * wz) * pv;
        }
        sx = group_sum<G>(sx);
        sy = group_sum<G>(sy);
        sz = group_sum<G>(sz);
        de = group_sum<G>(de);
        if(lane == 0) S.sr[2 * (size_t)n + i] = make_double4(sx / nui, sy / nui, sz / nui, de / nui);
    }
}

// ------------------------------------------------------------ time step, kick-drift
// dt = cflSound min_i h_i / max(c_s,i, 1e-10) (src/srgsph/sr_timestep.cpp:44-58)
__global__ void k_sr_dt(DevParams P, DevState S, int n, double* __restrict__ out)
{
    __shared__ double sm[SBLK / 32];
    double m = DBL_MAX;
    for(int i = blockIdx.x * SBLK + threadIdx.x; i < n; i += gridDim.x * SBLK) {
        const double cs = fmax(S.thermo[i].w, 1.0e-10);
        const double d = P.cfl_sound * S.vel[i].w / cs;
        if(d < m) m = d;
    }
    m = warp_min(m);
    if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if(threadIdx.x == 0) {
        for(int w = 1; w < SBLK / 32; ++w) m = fmin(m, sm[w]);
        atomic_min_pos(out, m);
    }
}

__device__ __forceinline__ void sr_store(const DevParams& P, DevState& S, int i, const SRKin& k, double N)
{
    double dens, pres;
    sr_eos(k.g, k.H, N, P.gamma, P.sr_c, dens, pres);
    double4 v = S.vel[i];
    v.x = k.vx;
    v.y = k.vy;
    v.z = k.vz;
    S.vel[i] = v;
    S.thermo[i] = make_double4(dens, pres, pres / ((P.gamma - 1.0) * dens), sr_sound(k.H, P.gamma));
    double4& aux = S.sr[(size_t)S.n + i];
    aux.z = k.g;
    aux.w = k.H;
}

// Solver::predict, SRGSPH branch: S, e a full step, positions drift with the
// half-step velocity, primitives at the full step.
__global__ void k_sr_predict(DevParams P, DevState S, int n, const double* __restrict__ dtp,
                             DevStatus* __restrict__ st)
{
    const int i = blockIdx.x * SBLK + threadIdx.x;
    if(i >= n) return;
    const double dt = *dtp;
    const double4 se = S.sr[i], rate = S.sr[2 * (size_t)n + i];
    const double N = S.sr[(size_t)n + i].x;
    const double hx = se.x + rate.x * (0.5 * dt), hy = se.y + rate.y * (0.5 * dt), hz = se.z + rate.z * (0.5 * dt);
    const double eh = se.w + rate.w * (0.5 * dt);
    const double4 sn = make_double4(se.x + rate.x * dt, se.y + rate.y * dt, se.z + rate.z * dt, se.w + rate.w * dt);
    S.sr[i] = sn;
    SRKin kh, kf;
    if(!sr_kin(hx, hy, hz, eh, P.gamma, P.sr_c, kh) || !sr_kin(sn.x, sn.y, sn.z, sn.w, P.gamma, P.sr_c, kf)) {
        st->sr_recovery = 1;
        return;
    }
    double4 p = S.pos[i];
    p.x = wrap(P, p.x + kh.vx * dt, 0);
    p.y = wrap(P, p.y + kh.vy * dt, 1);
    p.z = wrap(P, p.z + kh.vz * dt, 2);
    S.pos[i] = p;
    sr_store(P, S, i, kf, N);
    double dh, ph;
    sr_eos(kh.g, kh.H, N, P.gamma, P.sr_c, dh, ph);
    S.velp[i] = make_double4(kh.vx, kh.vy, kh.vz, ph / ((P.gamma - 1.0) * dh));
}

// Solver::correct, SRGSPH branch: S, e re-formed from the half step with the
// new rates, primitives recovered.
__global__ void k_sr_correct(DevParams P, DevState S, int n, const double* __restrict__ dtp,
                             DevStatus* __restrict__ st)
{
    const int i = blockIdx.x * SBLK + threadIdx.x;
    if(i >= n) return;
    const double dt = *dtp;
    const double4 se = S.sr[i], rate = S.sr[2 * (size_t)n + i];
    const double hx = se.x - rate.x * (0.5 * dt), hy = se.y - rate.y * (0.5 * dt), hz = se.z - rate.z * (0.5 * dt);
    const double eh = se.w - rate.w * (0.5 * dt);
    const double4 sn = make_double4(hx + rate.x * (0.5 * dt), hy + rate.y * (0.5 * dt), hz + rate.z * (0.5 * dt),
                                    eh + rate.w * (0.5 * dt));
    S.sr[i] = sn;
    SRKin k;
    if(!sr_kin(sn.x, sn.y, sn.z, sn.w, P.gamma, P.sr_c, k)) {
        st->sr_recovery = 1;
        return;
    }
    sr_store(P, S, i, k, S.sr[(size_t)n + i].x);
}

unsigned sr_grid(int n)
{
    const long long gpb = SBLK / SG;
    return (unsigned)std::max<long long>(1, std::min<long long>((n + gpb - 1) / gpb, 148LL * 16));
}

// The reference throws std::runtime_error from the Lorentz-factor solver
// (src/srgsph/sr_primitive_recovery.cpp:75); here the kernels flag it and the
// module reports it.
int sr_check(sphgpu_ctx* c)
{
    int flag = 0;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&flag, &c->d_status->sr_recovery, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if(flag) {
        const int zero = 0;
        SPHGPU_CUDA(c, cudaMemcpy(&c->d_status->sr_recovery, &zero, sizeof(int), cudaMemcpyHostToDevice));
        return fail(c, SPHGPU_ERR_SR_RECOVERY, "Lorentz factor solver did not converge");
    }
    return SPHGPU_OK;
}

}  // namespace

int sr_pre_interaction(sphgpu_ctx* c)
{
    const int n = c->n;
    if(c->first_pre) {
        stage_begin(c, SPHGPU_T_PRE);
        k_sr_initial_sml<<<grid_for(n, SBLK), SBLK, 0, c->stream>>>(c->dp, c->s, n);
        SPHGPU_LAUNCH_CHECK(c, "srgsph initial_smoothing");
        stage_end(c, SPHGPU_T_PRE, 1);
        c->first_pre = false;
    }
    const int rc_walk = gather_walk(c, false, 1.0);
    if(rc_walk < 0) return rc_walk;
    stage_begin(c, SPHGPU_T_PRE);
    k_sr_kin<<<grid_for(n, SBLK), SBLK, 0, c->stream>>>(c->dp, c->s, n, c->d_status);
    k_sr_pre_h<SG><<<sr_grid(n), SBLK, 0, c->stream>>>(c->dp, c->s, n, c->d_glist, c->d_gcount, (int)c->gcap);
    k_sr_pre_grad<SG><<<sr_grid(n), SBLK, 0, c->stream>>>(c->dp, c->s, n, c->d_glist, c->d_gcount, (int)c->gcap);
    SPHGPU_LAUNCH_CHECK(c, "srgsph PreInteraction");
    stage_end(c, SPHGPU_T_PRE, 3);
    int rc = sr_check(c);
    if(rc < 0) return rc;
    rc = tree_set_kernel(c);
    if(rc < 0) return rc;
    return rc_walk;
}

int sr_fluid_force(sphgpu_ctx* c)
{
    const int rc_walk = pair_walk(c);
    if(rc_walk < 0) return rc_walk;
    stage_begin(c, SPHGPU_T_FORCE);
    k_sr_force<SG><<<sr_grid(c->n), SBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_plist, c->d_pcount,
                                                         (int)c->pcap, c->d_dt);
    SPHGPU_LAUNCH_CHECK(c, "srgsph FluidForce");
    stage_end(c, SPHGPU_T_FORCE, 1);
    return rc_walk;
}

int sr_timestep(sphgpu_ctx* c)
{
    stage_begin(c, SPHGPU_T_TIMESTEP);
    const double big = DBL_MAX;
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_red, &big, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const unsigned nb = (unsigned)std::min<long long>(grid_for(c->n, SBLK), 148 * 4);
    k_sr_dt<<<nb, SBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_red);
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_dt, c->d_red, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    SPHGPU_LAUNCH_CHECK(c, "srgsph TimeStep");
    stage_end(c, SPHGPU_T_TIMESTEP, 1);
    return SPHGPU_OK;
}

int sr_predict(sphgpu_ctx* c)
{
    stage_begin(c, SPHGPU_T_PREDICT);
    k_sr_predict<<<grid_for(c->n, SBLK), SBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_dt, c->d_status);
    SPHGPU_LAUNCH_CHECK(c, "srgsph predict");
    stage_end(c, SPHGPU_T_PREDICT, 1);
    c->have_tree = false;
    return sr_check(c);
}

int sr_correct(sphgpu_ctx* c)
{
    stage_begin(c, SPHGPU_T_CORRECT);
    k_sr_correct<<<grid_for(c->n, SBLK), SBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_dt, c->d_status);
    SPHGPU_LAUNCH_CHECK(c, "srgsph correct");
    stage_end(c, SPHGPU_T_CORRECT, 1);
    return sr_check(c);
}

}  // namespace sphgpu
