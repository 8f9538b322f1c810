// pre.cu — PreInteraction::calculation for ssph, disph, gsph and gdisph.
//
// Reference: src/pre_interaction.cpp:39-283 (ssph, initial_smoothing,
// newton_raphson), src/disph/d_pre_interaction.cpp:21-230 (disph),
// src/gsph/g_pre_interaction.cpp:27-144 (gsph), src/gdisph/gd_pre_interaction.cpp:
// 29-280 (gdisph: the disph smoothing length, density and pressure, the gsph
// MUSCL gradients, a mass-weighted Balsara switch normalised by density, and
// without it the implicit alpha update weighted by mass x energy).
//
// A group of G lanes owns one particle and strides over its gather list
// (ELL row, coalesced index loads; neighbour state as 32-byte double4 loads
// that mostly hit L1/L2 because neighbours are close in octree order).
//   1. Newton-Raphson on h (<= 10 iterations, |dh| < 1e-4 (h + h_b)) over the
//      candidates with r < h, group-reduced each iteration;
//   2. one fused pass at the final h (disph: over the candidates the last
//      sweep kept, within (1 + 4e-4) of its h): density (and the DISPH number/pressure
//      sums), grad-h sums, max signal speed, neighbour count, the Balsara
//      div/curl sums and the GSPH MUSCL gradients — every quantity the
//      reference computes in separate loops over the same set {r < h};
//   3. per-particle epilogue (P, grad-h, Balsara, time-dependent alpha) and
//      the block-reduced minimum of h / v_sig.
// The set predicates (r computed from the unfused FP64 r^2, r < h) match the
// reference exactly; sums are taken in a different order than the
// reference's distance-sorted loop, so results agree to rounding.
// T = double: plain FP64 form.  T = float: pair arithmetic and sums in FP32
// (mixed form); h, its Newton update and the predicates stay FP64.
// Loading the next neighbour's position one iteration ahead as well (not only
// its index) was measured slower: shear 1 M, 5.38 ms against 4.78 ms (FP64),
// 4.29 against 3.67 ms (mixed); the extra live double4 adds spills.
#include <cfloat>
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr double AREA3 = 4.0 * 3.14159265358979323846 / 3.0;  // A for DIM = 3
constexpr int PBLK = 256;

__device__ __forceinline__ double exact_r(const DevParams& P, double xi, double yi, double zi, double4 pj,
                                          Vec3d& d)
{
    d = rij(P, xi, yi, zi, pj.x, pj.y, pj.z);
    return sqrt(abs2x(d));
}

// The Newton sweep's pair test and distance: true when r < h exactly as the
// reference decides it (root_lt on the unfused FP64 r^2); r in the sweep's
// precision (FP64: rsqrt-based, FP32: from the FP32 r^2).
__device__ __forceinline__ bool sweep_r(double r2, double h, double& r)
{
    double rinv;
    return pair_within(r2, h, r, rinv);
}
__device__ __forceinline__ bool sweep_r(double r2, double h, float& r)
{
    if(!root_lt(r2, h)) return false;
    const float r2f = (float)r2;
    r = r2f > 0.f ? r2f * rsqrtf(r2f) : 0.f;
    return true;
}

// Minimum resident blocks per SM (caps registers; measured on B200).  The
// FP64 forms of disph, gsph and gdisph take 2 (no spills): 8.78 M sphere
// disph 40.3 -> 34.6 ms, 2 M tubes gsph 4.5 -> 3.7, gdisph 6.7 -> 4.3 ms; the
// 1 M shear layer no slower.  FP32: disph 3 (30.6 -> 28.7 ms), gsph / gdisph 3
// (2 is slower), ssph 4.
template <typename T, int TYPE>
constexpr int pre_min_blocks()
{
    if(sizeof(T) == sizeof(double)) return TYPE == SPHGPU_SSPH ? 3 : 2;
    return TYPE == SPHGPU_SSPH ? 4 : 3;
}

// skin_delta > 0: the lists are skin lists (supersets of the gather lists);
// a particle whose h reaches R - skin_delta (R = its gather radius, the sml
// the walk left) takes only exact members (gather_member).
template <typename T, int G, int TYPE>
__global__ void __launch_bounds__(PBLK, (pre_min_blocks<T, TYPE>())) k_pre(DevParams P, DevState S, int n, const int* __restrict__ list,
                                              const int* __restrict__ count, int cap, const double* __restrict__ dtp,
                                              double* __restrict__ hvs, DevStatus* __restrict__ st, DevTree Tr,
                                              double skin_delta, int* __restrict__ scratch, int scap)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * PBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * PBLK) >> 5;
    const double dt = *dtp;
    constexpr bool gdisph = TYPE == SPHGPU_GDISPH;
    const bool disph = TYPE == SPHGPU_DISPH || gdisph, gsph = TYPE == SPHGPU_GSPH;
    // AV switch sums weighted by m_j u_j and normalised by (gamma - 1) / P
    // (disph; gdisph without the Balsara switch), else by m_j and 1 / rho
    const bool av_energy = disph && !(gdisph && P.balsara);
    double hv_min = DBL_MAX;
    unsigned nonconv = 0;
    unsigned n_cand = 0, n_newton = 0, n_pairs = 0, n_list = 0;  // work counters of this lane

    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        const bool valid = i < n;
        const int cnt = valid ? min(count[i], cap) : 0;
        const int* li = list + (size_t)(valid ? i : 0) * (size_t)cap;
        const double4 pi = valid ? S.pos[i] : make_double4(0, 0, 0, 0);
        const double4 vi = valid ? S.vel[i] : make_double4(0, 0, 0, 1);
        const double4 ti = valid ? S.thermo[i] : make_double4(1, 0, 0, 0);
        const double sml0 = vi.w;

        // ---- 1. smoothing length (src/pre_interaction.cpp:227-283,
        //         src/disph/d_pre_interaction.cpp:174-230)
        double h = sml0;
        // disph: each sweep also keeps, per lane and in the lane's own order,
        // the candidates within (1 + 4e-4) h in a scratch row; after a
        // converged sweep (|h_new - h| < 1e-4 (h_new + h), so h_new <
        // (1 + 2.0003e-4) h) they hold every pair of the fused pass, which
        // then reads them instead of the whole list (8.78 M sphere: pre 31.8
        // -> 30.8 ms FP64, 27.4 -> 24.1 ms FP32; the gsph and gdisph bodies
        // spill with it and run slower)
        constexpr bool keep = TYPE == SPHGPU_DISPH;
        int* srow = scratch + (size_t)(valid ? i : 0) * (size_t)scap;
        int nk = 0;
        bool conv = false;
        if(P.iterative) {
            h = sml0 / P.ratio;
            const double b = disph ? P.nngb / AREA3 : pi.w * P.nngb / AREA3;
            for(int it = 0; it < 10; ++it) {
                const double hb = h;
                T d = 0, dd = 0;
                const KernH<T> kh(P.kernel, (T)h);
                const bool exact = skin_delta > 0.0 && !(h < sml0 - skin_delta);
                const double hk = h * (1.0 + 4e-4), keep2 = hk * hk;
                nk = 0;
                auto visit = [&](const double4& pj, int jc) {
                    const double r2 = abs2x(rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z));
                    if constexpr(keep) {
                        if(r2 < keep2) srow[lane + G * nk++] = jc;
                    }
                    T rT;
                    if(sweep_r(r2, h, rT) && (!exact || gather_member(P, Tr, pi.x, pi.y, pi.z, sml0, skin_delta, jc, r2))) {
                        ++n_newton;
                        const T w = kh.w(rT);
                        const T dh = kh.dhw(rT);
                        if(disph) {
                            d += w;
                            dd += dh;
                        } else {
                            d += (T)pj.w * w;
                            dd += (T)pj.w * dh;
                        }
                    }
                };
                // two candidates per iteration (the same per-lane order), their
                // indices fetched an iteration ahead: two position loads in
                // flight, neither waiting on the list load (8.78 M sphere:
                // 34.9 -> 32.5 ms FP64)
                int ja = lane < cnt ? __ldg(&li[lane]) : 0;
                int jb = lane + G < cnt ? __ldg(&li[lane + G]) : 0;
                n_cand += lane < cnt ? (unsigned)((cnt - lane + G - 1) / G) : 0u;
                for(int k = lane; k < cnt; k += 2 * G) {
                    const int ca = ja, cb = jb;  // cb is a valid index even past the list end
                    const bool two = k + G < cnt;
                    if(k + 2 * G < cnt) ja = __ldg(&li[k + 2 * G]);
                    if(k + 3 * G < cnt) jb = __ldg(&li[k + 3 * G]);
                    const double4 pa = ldg4(&S.pos[ca]);
                    const double4 pb = ldg4(&S.pos[cb]);
                    visit(pa, ca);
                    if(two) visit(pb, cb);
                }
                const double ds = (double)group_sum<G>(d), dds = (double)group_sum<G>(dd);
                const double h3 = h * h * h;
                const double f = ds * h3 - b;
                const double df = dds * h3 + 3 * ds * (h * h);
                h -= f / df;
                if(fabs(h - hb) < (h + hb) * 1e-4) {
                    conv = true;
                    break;
                }
            }
            if(!conv) {
                h = sml0 / P.ratio;
                if(valid && lane == 0) ++nonconv;
            }
        }

        // ---- 2. fused pass over {r < h}
        const KernH<T> kh(P.kernel, (T)h);
        T dens = 0, dhd = 0, ni = 0, pres = 0, dhp = 0, dhn = 0;
        T divv = 0, rx = 0, ry = 0, rz = 0;
        T gd[3] = {0, 0, 0}, gu[3] = {0, 0, 0}, gv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double vsig = ti.w * 2.0;
        int nn = 0;
        const bool need_av = !gsph && (P.balsara || P.td_av);
        const bool need_grad = (gsph || gdisph) && P.gsph2;
        const bool exact = skin_delta > 0.0 && !(h < sml0 - skin_delta);
        n_list += lane < cnt ? (unsigned)((cnt - lane + G - 1) / G) : 0u;
        const bool kept = keep && conv;
        n_cand += kept ? (unsigned)nk : (lane < cnt ? (unsigned)((cnt - lane + G - 1) / G) : 0u);
        auto visit = [&](const double4& pj, int j) {
            const Vec3d dv = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double r2 = abs2x(dv);
            double r, rinv;
            if constexpr(sizeof(T) == sizeof(float)) {
                // the set predicate in FP64, the distance in FP32 (mixed form)
                if(!root_lt(r2, h)) return;
                const float r2f = (float)r2;
                const float rif = r2f > 0.f ? rsqrtf(r2f) : 0.f;
                r = (double)(r2f * rif);
                rinv = (double)rif;
            } else {
                if(!pair_within(r2, h, r, rinv)) return;
            }
            if(exact && !gather_member(P, Tr, pi.x, pi.y, pi.z, sml0, skin_delta, j, r2)) return;
            ++nn;
            // coherent loads: this kernel writes vel.w and thermo.x, .y of every
            // particle (the components read here, velocity, u and c_s, it
            // does not change)
            const double4 vj = S.vel[j];
            const double4 tj = S.thermo[j];
            const T rT = (T)r;
            const T w = kh.w(rT);
            const T mj = (T)pj.w;
            if(disph) {
                const T dh = kh.dhw(rT);
                const T uj = (T)tj.z;
                dens += mj * w;
                ni += w;
                pres += mj * uj * w;
                dhp += mj * uj * dh;
                dhn += dh;
            } else {
                dens += mj * w;
                if(!gsph) dhd += mj * kh.dhw(rT);
            }
            if(i != j) {
                const double vr = dv.x * (vi.x - vj.x) + dv.y * (vi.y - vj.y) + dv.z * (vi.z - vj.z);
                // coincident particles (r = 0): the reference's vr / r is
                // 0 / 0, a NaN that never raises v_sig (+-inf if r underflowed)
                const double v = r > 0.0 ? ti.w + tj.w - 3.0 * vr * rinv
                                         : (vr < 0.0 ? (double)INFINITY : -(double)INFINITY);
                if(v > vsig) vsig = v;
            }
            if(need_av || need_grad) {
                const T c = kh.dwc(rT, (T)rinv);
                const T dwx = (T)dv.x * c, dwy = (T)dv.y * c, dwz = (T)dv.z * c;
                const T vx = (T)(vi.x - vj.x), vy = (T)(vi.y - vj.y), vz = (T)(vi.z - vj.z);
                if(need_av) {
                    const T wgt = av_energy ? mj * (T)tj.z : mj;
                    divv -= wgt * (vx * dwx + vy * dwy + vz * dwz);
                    rx += (vy * dwz - vz * dwy) * wgt;
                    ry += (vz * dwx - vx * dwz) * wgt;
                    rz += (vx * dwy - vy * dwx) * wgt;
                }
                if(need_grad) {
                    const T du = mj * (T)(tj.z - ti.z);
                    gd[0] += dwx * mj;
                    gd[1] += dwy * mj;
                    gd[2] += dwz * mj;
                    gu[0] += dwx * du;
                    gu[1] += dwy * du;
                    gu[2] += dwz * du;
                    // dv[k] += dw * (m_j (v_j[k] - v_i[k]))
                    const T m0 = -mj * vx, m1 = -mj * vy, m2 = -mj * vz;
                    gv[0] += dwx * m0;
                    gv[1] += dwy * m0;
                    gv[2] += dwz * m0;
                    gv[3] += dwx * m1;
                    gv[4] += dwy * m1;
                    gv[5] += dwz * m1;
                    gv[6] += dwx * m2;
                    gv[7] += dwy * m2;
                    gv[8] += dwz * m2;
                }
            }
        };
        if(kept) {
            // the lane's kept candidates, in its own order (the same sums)
            int m = 0;
            for(; m + 1 < nk; m += 2) {
                const int ca = srow[lane + G * m], cb = srow[lane + G * (m + 1)];
                const double4 pa = ldg4(&S.pos[ca]);
                const double4 pb = ldg4(&S.pos[cb]);
                visit(pa, ca);
                visit(pb, cb);
            }
            if(m < nk) {
                const int ca = srow[lane + G * m];
                visit(ldg4(&S.pos[ca]), ca);
            }
        } else if constexpr(sizeof(T) == sizeof(double) && TYPE == SPHGPU_DISPH) {
            // two candidates per iteration, as in the sweep (8.78 M sphere
            // 32.4 -> 31.7 ms; slower for the other instantiations, whose
            // larger bodies then spill)
            int ja = lane < cnt ? __ldg(&li[lane]) : 0;
            int jb = lane + G < cnt ? __ldg(&li[lane + G]) : 0;
            for(int k = lane; k < cnt; k += 2 * G) {
                const int ca = ja, cb = jb;  // cb is a valid index even past the list end
                const bool two = k + G < cnt;
                if(k + 2 * G < cnt) ja = __ldg(&li[k + 2 * G]);
                if(k + 3 * G < cnt) jb = __ldg(&li[k + 3 * G]);
                const double4 pa = ldg4(&S.pos[ca]);
                const double4 pb = ldg4(&S.pos[cb]);
                visit(pa, ca);
                if(two) visit(pb, cb);
            }
        } else {
            // the next candidate's index is fetched one iteration ahead
            int jn = lane < cnt ? __ldg(&li[lane]) : 0;
            for(int k = lane; k < cnt; k += G) {
                const int j = jn;
                if(k + G < cnt) jn = __ldg(&li[k + G]);
                visit(ldg4(&S.pos[j]), j);
            }
        }
        n_pairs += (unsigned)nn;
        const double densS = (double)group_sum<G>(dens);
        nn = group_sum<G>(nn);
        vsig = group_max<G>(vsig);
        double dhdS = 0, niS = 0, presS = 0, dhpS = 0, dhnS = 0;
        if(disph) {
            niS = (double)group_sum<G>(ni);
            presS = (double)group_sum<G>(pres);
            dhpS = (double)group_sum<G>(dhp);
            dhnS = (double)group_sum<G>(dhn);
        } else if(!gsph) {
            dhdS = (double)group_sum<G>(dhd);
        }
        double divS = 0, rxS = 0, ryS = 0, rzS = 0;
        if(need_av) {
            divS = (double)group_sum<G>(divv);
            rxS = (double)group_sum<G>(rx);
            ryS = (double)group_sum<G>(ry);
            rzS = (double)group_sum<G>(rz);
        }
        double gdS[3], guS[3], gvS[9];
        if(need_grad) {
#pragma unroll
            for(int k = 0; k < 3; ++k) {
                gdS[k] = (double)group_sum<G>(gd[k]);
                guS[k] = (double)group_sum<G>(gu[k]);
            }
#pragma unroll
            for(int k = 0; k < 9; ++k) gvS[k] = (double)group_sum<G>(gv[k]);
        }

        // ---- 3. epilogue (lane 0 of the group writes)
        if(!valid || lane != 0) continue;
        const double gamma = P.gamma;
        const double ui = ti.z, ci = ti.w;
        double pres_i;
        double4 vs = S.visc[i];
        if(disph) {
            pres_i = (gamma - 1.0) * presS;
            vs.z = h / (3 * niS) * dhpS / (1.0 + h / (3 * niS) * dhnS);
        } else {
            pres_i = (gamma - 1.0) * densS * ui;
            if(!gsph) vs.z = 1.0 / (1.0 + h / (3 * densS) * dhdS);
        }
        S.thermo[i] = make_double4(densS, pres_i, ui, ci);
        S.vel[i].w = h;
        S.nbr[i] = nn;
        const double hv = h / vsig;
        if(hv < hv_min) hv_min = hv;
        if(need_av) {
            // Balsara switch and time-dependent alpha (src/pre_interaction.cpp:115-161,
            // src/disph/d_pre_interaction.cpp:106-154)
            double dv_ = divS, r0 = rxS, r1 = ryS, r2 = rzS;
            if(av_energy) {
                const double pinv = (gamma - 1.0) / pres_i;
                dv_ *= pinv;
                r0 *= pinv;
                r1 *= pinv;
                r2 *= pinv;
            } else {
                dv_ /= densS;
                r0 /= densS;
                r1 /= densS;
                r2 /= densS;
            }
            if(P.balsara) {
                const double rot = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
                vs.y = fabs(dv_) / (fabs(dv_) + rot + 1e-4 * ci / h);
                if(P.td_av) {
                    const double tau = P.eps_av * ci / h;
                    const double da = (-(vs.x - P.alpha_min) * tau + fmax(-dv_, 0.0) * (P.alpha_max - vs.x)) * dt;
                    vs.x += da;
                }
            } else {
                const double tau = P.eps_av * ci / h;
                const double s = fmax(-dv_, 0.0);
                vs.x = (vs.x + dt * tau * P.alpha_min + s * dt * P.alpha_max) / (1.0 + dt * tau + s * dt);
            }
        }
        S.visc[i] = vs;
        if(need_grad) {
            // MUSCL gradients (src/gsph/g_pre_interaction.cpp:112-136)
            const double gm1 = gamma - 1.0, rinv = 1.0 / densS;
            const double g15[15] = {gdS[0],
                                    gdS[1],
                                    gdS[2],
                                    (gdS[0] * ui + guS[0]) * gm1,
                                    (gdS[1] * ui + guS[1]) * gm1,
                                    (gdS[2] * ui + guS[2]) * gm1,
                                    gvS[0] * rinv,
                                    gvS[1] * rinv,
                                    gvS[2] * rinv,
                                    gvS[3] * rinv,
                                    gvS[4] * rinv,
                                    gvS[5] * rinv,
                                    gvS[6] * rinv,
                                    gvS[7] * rinv,
                                    gvS[8] * rinv};
            S.grad[i] = make_double4(g15[0], g15[1], g15[2], g15[3]);
            S.grad[(size_t)n + i] = make_double4(g15[4], g15[5], g15[6], g15[7]);
            S.grad[2 * (size_t)n + i] = make_double4(g15[8], g15[9], g15[10], g15[11]);
            S.grad[3 * (size_t)n + i] = make_double4(g15[12], g15[13], g15[14], 0.0);
        }
    }
    // block reductions: min h / v_sig, Newton fallbacks
    __shared__ double s_min[PBLK / 32];
    __shared__ unsigned s_nc[PBLK / 32];
    hv_min = warp_min(hv_min);
    for(int o = 16; o > 0; o >>= 1) nonconv += __shfl_xor_sync(FULL_MASK, nonconv, o);
    if((threadIdx.x & 31) == 0) {
        s_min[threadIdx.x >> 5] = hv_min;
        s_nc[threadIdx.x >> 5] = nonconv;
    }
    __syncthreads();
    if(threadIdx.x == 0) {
        double m = s_min[0];
        unsigned c = s_nc[0];
        for(int w = 1; w < PBLK / 32; ++w) {
            m = fmin(m, s_min[w]);
            c += s_nc[w];
        }
        if(m < DBL_MAX) atomic_min_pos(hvs, m);
        if(c) atomicAdd(&st->newton_nonconv, (unsigned long long)c);
    }
    block_count(&st->pre_cand, n_cand);
    block_count(&st->pre_newton_pairs, n_newton);
    block_count(&st->pre_pairs, n_pairs);
    block_count(&st->pre_list, n_list);
}

// PreInteraction::initial_smoothing (src/pre_interaction.cpp:171-215):
// density at the guessed h over {r < h}.
template <typename T, int G>
__global__ void __launch_bounds__(PBLK) k_initial_density(DevParams P, DevState S, int n,
                                                          const int* __restrict__ list,
                                                          const int* __restrict__ count, int cap)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const long long warp = ((long long)blockIdx.x * PBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * PBLK) >> 5;
    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        const bool valid = i < n;
        const int cnt = valid ? min(count[i], cap) : 0;
        const int* li = list + (size_t)(valid ? i : 0) * (size_t)cap;
        const double4 pi = valid ? S.pos[i] : make_double4(0, 0, 0, 0);
        const double h = valid ? S.vel[i].w : 1.0;
        const KernH<T> kh(P.kernel, (T)h);
        T d = 0;
        for(int k = lane; k < cnt; k += G) {
            const double4 pj = S.pos[li[k]];
            Vec3d dv;
            const double r = exact_r(P, pi.x, pi.y, pi.z, pj, dv);
            if(r < h) d += (T)pj.w * kh.w((T)r);
        }
        const double ds = (double)group_sum<G>(d);
        if(valid && lane == 0) S.thermo[i].x = ds;
    }
}

constexpr int GROUP = 4;

unsigned pre_grid(int n)
{
    const long long groups_per_block = PBLK / GROUP;
    long long blocks = (n + groups_per_block - 1) / groups_per_block;
    const long long cap = 148LL * 8 * 4;
    return (unsigned)std::max<long long>(1, std::min(blocks, cap));
}

template <typename T>
void launch_pre(sphgpu_ctx* c)
{
    const unsigned grid = pre_grid(c->n);
    const double sd = c->skin_valid ? c->skin_delta_now : 0.0;
    const int type = c->prm.sph_type;
    if(type == SPHGPU_DISPH) {
        k_pre<T, GROUP, SPHGPU_DISPH><<<grid, PBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_glist, c->d_gcount,
                                                                    (int)c->gcap, c->d_dt, c->d_hvs, c->d_status, c->t, sd,
                                                                   c->d_plist, (int)c->pcap);
    } else if(type == SPHGPU_GSPH) {
        k_pre<T, GROUP, SPHGPU_GSPH><<<grid, PBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_glist, c->d_gcount,
                                                                   (int)c->gcap, c->d_dt, c->d_hvs, c->d_status, c->t, sd,
                                                                   c->d_plist, (int)c->pcap);
    } else if(type == SPHGPU_GDISPH) {
        k_pre<T, GROUP, SPHGPU_GDISPH><<<grid, PBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_glist, c->d_gcount,
                                                                     (int)c->gcap, c->d_dt, c->d_hvs, c->d_status, c->t, sd,
                                                                   c->d_plist, (int)c->pcap);
    } else {
        k_pre<T, GROUP, SPHGPU_SSPH><<<grid, PBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_glist, c->d_gcount,
                                                                   (int)c->gcap, c->d_dt, c->d_hvs, c->d_status, c->t, sd,
                                                                   c->d_plist, (int)c->pcap);
    }
}

}  // namespace

int pre_interaction(sphgpu_ctx* c)
{
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "PreInteraction before tree make");
    if(c->prm.sph_type == SPHGPU_SRGSPH) return sr_pre_interaction(c);
    int rc_walk = SPHGPU_OK;
    const bool mixed = c->prm.precision == SPHGPU_MIXED;
    if(c->first_pre) {
        // initial_smoothing: h from the initial density, no kernel ratio
        int rc = gather_walk(c, true, 1.0);
        if(rc < 0) return rc;
        stage_begin(c, SPHGPU_T_PRE);
        if(mixed) {
            k_initial_density<float, GROUP><<<pre_grid(c->n), PBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_glist,
                                                                                    c->d_gcount, (int)c->gcap);
        } else {
            k_initial_density<double, GROUP><<<pre_grid(c->n), PBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_glist,
                                                                                     c->d_gcount, (int)c->gcap);
        }
        SPHGPU_LAUNCH_CHECK(c, "initial_smoothing");
        stage_end(c, SPHGPU_T_PRE, 1);
        c->first_pre = false;
    }
    rc_walk = gather_lists(c, c->dp.ratio);
    if(rc_walk < 0) return rc_walk;
    int rcs = save_gather_radius(c);
    if(rcs < 0) return rcs;
    // the pair-list buffer is the sweeps' scratch (the pair lists are built after)
    if(c->pcap < c->gcap && (rcs = ensure_list_capacity(c, 1, c->gcap)) < 0) return rcs;
    stage_begin(c, SPHGPU_T_PRE);
    const double big = DBL_MAX;
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_hvs, &big, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if(mixed) launch_pre<float>(c);
    else launch_pre<double>(c);
    SPHGPU_LAUNCH_CHECK(c, "PreInteraction");
    stage_end(c, SPHGPU_T_PRE, 1);
    int rc = tree_set_kernel(c);
    if(rc < 0) return rc;
    rc = build_force_lists(c);
    if(rc < 0) return rc;
    return rc_walk;
}

}  // namespace sphgpu
