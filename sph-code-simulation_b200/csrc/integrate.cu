// integrate.cu — TimeStep::calculation, Solver::predict / correct and
// Solver::compute_total_energies.
//
// Reference: src/timestep.cpp:18-38, src/solver.cpp:1046-1061 (predict),
// :1104-1112 (correct), :1149-1175 (energies).  All FP64 in both forms; this
// file builds with -fmad=false so the kick-drift is bit-identical to the
// reference's on identical inputs.  dt lives in device memory: predict and
// correct read it there, so a whole step runs without a host round trip.
#include <cfloat>
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int IBLK = 256;

__global__ void k_dt_partial(DevState S, int n, double cfl_force, double* __restrict__ out)
{
    __shared__ double sm[IBLK / 32];
    double m = DBL_MAX;
    for(int i = blockIdx.x * IBLK + threadIdx.x; i < n; i += gridDim.x * IBLK) {
        const double4 a = S.acc[i];
        const double aa = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        if(aa > 0.0) {
            const double d = cfl_force * sqrt(S.vel[i].w / aa);
            if(d < m) m = d;
        }
    }
    m = warp_min(m);
    if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if(threadIdx.x == 0) {
        for(int w = 1; w < IBLK / 32; ++w) m = fmin(m, sm[w]);
        m = fmin(m, sm[0]);
        atomic_min_pos(out, m);
    }
}

__global__ void k_dt_final(const double* __restrict__ dtmin, const double* __restrict__ hvs, double cfl_sound,
                           double* __restrict__ dt)
{
    const double ds = cfl_sound * *hvs;
    const double df = *dtmin;
    *dt = df < ds ? df : ds;  // std::min(dt_sound, dt_force)
}

__device__ __forceinline__ double wrap(const DevParams& P, double x, int k)
{
    if(!P.periodic) return x;
    if(x < P.lo[k]) return x + P.range[k];
    if(x > P.hi[k]) return x - P.range[k];
    return x;
}

__global__ void k_predict(DevParams P, DevState S, int n, const double* __restrict__ dtp)
{
    const int i = blockIdx.x * IBLK + threadIdx.x;
    if(i >= n) return;
    const double dt = *dtp, hdt = 0.5 * dt;
    const double cs = P.gamma * (P.gamma - 1.0);
    double4 p = S.pos[i], v = S.vel[i];
    const double4 a = S.acc[i];
    double4 t = S.thermo[i];
    double4 vp;
    vp.x = v.x + a.x * hdt;
    vp.y = v.y + a.y * hdt;
    vp.z = v.z + a.z * hdt;
    vp.w = t.z + a.w * hdt;
    p.x = wrap(P, p.x + vp.x * dt, 0);
    p.y = wrap(P, p.y + vp.y * dt, 1);
    p.z = wrap(P, p.z + vp.z * dt, 2);
    v.x = v.x + a.x * dt;
    v.y = v.y + a.y * dt;
    v.z = v.z + a.z * dt;
    t.z = t.z + a.w * dt;
    t.w = sqrt(cs * t.z);
    S.pos[i] = p;
    S.vel[i] = v;
    S.velp[i] = vp;
    S.thermo[i] = t;
}

__global__ void k_correct(DevParams P, DevState S, int n, const double* __restrict__ dtp)
{
    const int i = blockIdx.x * IBLK + threadIdx.x;
    if(i >= n) return;
    const double hdt = 0.5 * *dtp;
    const double cs = P.gamma * (P.gamma - 1.0);
    double4 v = S.vel[i];
    const double4 vp = S.velp[i], a = S.acc[i];
    double4 t = S.thermo[i];
    v.x = vp.x + a.x * hdt;
    v.y = vp.y + a.y * hdt;
    v.z = vp.z + a.z * hdt;
    t.z = vp.w + a.w * hdt;
    t.w = sqrt(cs * t.z);
    S.vel[i] = v;
    S.thermo[i] = t;
}

// K, U, W and momentum: per-block partials in a fixed order, then one block.
constexpr int EBLK = 256;
__global__ void k_energy_partial(DevState S, int n, int gravity, double* __restrict__ part)
{
    __shared__ double sm[6][EBLK];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for(int i = blockIdx.x * EBLK + threadIdx.x; i < n; i += gridDim.x * EBLK) {
        const double m = S.pos[i].w;
        const double4 v = S.vel[i];
        acc[0] += 0.5 * m * (v.x * v.x + v.y * v.y + v.z * v.z);
        acc[1] += m * S.thermo[i].z;
        if(gravity) acc[2] += 0.5 * m * S.visc[i].w;
        acc[3] += m * v.x;
        acc[4] += m * v.y;
        acc[5] += m * v.z;
    }
    for(int k = 0; k < 6; ++k) sm[k][threadIdx.x] = acc[k];
    __syncthreads();
    for(int s = EBLK / 2; s > 0; s >>= 1) {
        if(threadIdx.x < s) {
            for(int k = 0; k < 6; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + s];
        }
        __syncthreads();
    }
    if(threadIdx.x == 0) {
        for(int k = 0; k < 6; ++k) part[blockIdx.x * 6 + k] = sm[k][0];
    }
}

__global__ void k_energy_final(const double* __restrict__ part, int nb, double* __restrict__ out)
{
    if(threadIdx.x != 0) return;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for(int b = 0; b < nb; ++b) {
        for(int k = 0; k < 6; ++k) acc[k] += part[b * 6 + k];
    }
    for(int k = 0; k < 6; ++k) out[k] = acc[k];
}

}  // namespace

int timestep(sphgpu_ctx* c)
{
    if(c->prm.sph_type == SPHGPU_SRGSPH) return sr_timestep(c);
    stage_begin(c, SPHGPU_T_TIMESTEP);
    const double big = DBL_MAX;
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_red, &big, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const unsigned nb = (unsigned)std::min<long long>(grid_for(c->n, IBLK), 148 * 4);
    k_dt_partial<<<nb, IBLK, 0, c->stream>>>(c->s, c->n, c->prm.cfl_force, c->d_red);
    k_dt_final<<<1, 1, 0, c->stream>>>(c->d_red, c->d_hvs, c->prm.cfl_sound, c->d_dt);
    SPHGPU_LAUNCH_CHECK(c, "TimeStep");
    stage_end(c, SPHGPU_T_TIMESTEP, 2);
    return SPHGPU_OK;
}

int predict(sphgpu_ctx* c)
{
    if(c->prm.sph_type == SPHGPU_SRGSPH) return sr_predict(c);
    stage_begin(c, SPHGPU_T_PREDICT);
    k_predict<<<grid_for(c->n, IBLK), IBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_dt);
    SPHGPU_LAUNCH_CHECK(c, "predict");
    stage_end(c, SPHGPU_T_PREDICT, 1);
    c->have_tree = false;  // positions moved
    return SPHGPU_OK;
}

int correct(sphgpu_ctx* c)
{
    if(c->prm.sph_type == SPHGPU_SRGSPH) return sr_correct(c);
    stage_begin(c, SPHGPU_T_CORRECT);
    k_correct<<<grid_for(c->n, IBLK), IBLK, 0, c->stream>>>(c->dp, c->s, c->n, c->d_dt);
    SPHGPU_LAUNCH_CHECK(c, "correct");
    stage_end(c, SPHGPU_T_CORRECT, 1);
    return SPHGPU_OK;
}

int energies(sphgpu_ctx* c, double* out6)
{
    const int nb = (int)std::min<long long>(grid_for(c->n, EBLK), 1024);
    k_energy_partial<<<nb, EBLK, 0, c->stream>>>(c->s, c->n, c->prm.use_gravity, c->d_red + 8);
    k_energy_final<<<1, 32, 0, c->stream>>>(c->d_red + 8, nb, c->d_red);
    SPHGPU_LAUNCH_CHECK(c, "energies");
    SPHGPU_CUDA(c, cudaMemcpyAsync(out6, c->d_red, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return SPHGPU_OK;
}

}  // namespace sphgpu
