// relax.cu — the Lane-Emden relaxation step.
//
// Reference: Solver's relaxation loop (src/solver.cpp:779-829) and
// LaneEmdenRelaxation (src/relaxation/lane_emden_relaxation.cpp:35-138,
// src/relaxation/lane_emden_data.cpp:66-113).  One step: tree, PreInteraction,
// FluidForce, GravityForce (when on); subtract from every acceleration the
// analytic Lane-Emden equilibrium acceleration
//   a_r = -(K gamma n / alpha) theta(xi)^(gamma - 1) dtheta/dxi(xi),  n = 1.5,
//   xi = |x| / alpha, theta and dtheta linearly interpolated in the caller's
//   table (zero outside xi_1, at the centre, or where theta <= 0);
// TimeStep's dt times 0.1; v = 0 and x += a dt^2 / 2 with the periodic wrap.
// The set-up before the loop (sound speeds, src/solver.cpp:744-752) runs on
// the first step.  Unfused FP64 (-fmad=false) as the reference; pow is
// CUDA's, so accelerations agree with the reference to rounding.
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int RBLK = 256;

// LaneEmdenData::get_theta / dtheta_dxi: lower_bound, then linear interpolation
__device__ __forceinline__ double table_at(const double* __restrict__ x, const double* __restrict__ y, int64_t np,
                                           double xi)
{
    int64_t lo = 0, hi = np;
    for(int it = 0; it < 64 && lo < hi; ++it) {
        const int64_t mid = (lo + hi) >> 1;
        if(x[mid] < xi) lo = mid + 1;
        else hi = mid;
    }
    if(lo >= np) return 0.0;
    if(lo == 0) return y[0];
    const double frac = (xi - x[lo - 1]) / (x[lo] - x[lo - 1]);
    return y[lo - 1] * (1.0 - frac) + y[lo] * frac;
}

__global__ void k_relax_sound(DevParams P, DevState S, int n)
{
    const int i = blockIdx.x * RBLK + threadIdx.x;
    if(i >= n) return;
    const double cs = P.gamma * (P.gamma - 1.0);
    S.thermo[i].w = sqrt(cs * S.thermo[i].z);
}

__global__ void k_relax_apply(DevParams P, DevState S, int n, const double* __restrict__ tab, int64_t np, double xi1,
                              double alpha, double K)
{
    const int i = blockIdx.x * RBLK + threadIdx.x;
    if(i >= n) return;
    const double4 p = S.pos[i];
    const double r = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    if(r < 1e-12) return;
    const double xi = r / alpha;
    if(xi >= xi1) return;
    const double theta = xi <= 0.0 ? 1.0 : table_at(tab, tab + np, np, xi);
    const double dtheta = xi <= 0.0 ? 0.0 : table_at(tab, tab + 2 * np, np, xi);
    if(theta <= 0.0) return;
    const double prefactor = K * P.gamma * 1.5 / alpha;
    const double a_r = -prefactor * pow(theta, P.gamma - 1.0) * dtheta;
    const double rinv = 1.0 / r;
    double4 a = S.acc[i];
    a.x -= -a_r * p.x * rinv;
    a.y -= -a_r * p.y * rinv;
    a.z -= -a_r * p.z * rinv;
    S.acc[i] = a;
}

__device__ __forceinline__ double wrap_axis(const DevParams& P, double x, int k)
{
    if(!P.periodic) return x;
    if(x < P.lo[k]) return x + P.range[k];
    if(x > P.hi[k]) return x - P.range[k];
    return x;
}

__global__ void k_relax_move(DevParams P, DevState S, int n, const double* __restrict__ dtp, double* __restrict__ dtr)
{
    const int i = blockIdx.x * RBLK + threadIdx.x;
    const double d = *dtp * 0.1;
    if(i == 0) *dtr = d;
    if(i >= n) return;
    double4 p = S.pos[i], v = S.vel[i];
    const double4 a = S.acc[i];
    v.x = 0.0;
    v.y = 0.0;
    v.z = 0.0;
    p.x = wrap_axis(P, p.x + 0.5 * a.x * d * d, 0);
    p.y = wrap_axis(P, p.y + 0.5 * a.y * d * d, 1);
    p.z = wrap_axis(P, p.z + 0.5 * a.z * d * d, 2);
    S.pos[i] = p;
    S.vel[i] = v;
}

}  // namespace

}  // namespace sphgpu

using namespace sphgpu;

extern "C" int sphgpu_relax_step(sphgpu_ctx* c, const sphgpu_lane_emden* le, int first, double* dt_relax)
{
    if(!c) return SPHGPU_ERR_ARG;
    if(c->n <= 0) return fail(c, SPHGPU_ERR_STATE, "no particles uploaded");
    if(!le || !le->xi || !le->theta || !le->dtheta || le->npts < 2 || !(le->alpha_scaling > 0.0))
        return fail(c, SPHGPU_ERR_ARG, "relax_step: the Lane-Emden table needs >= 2 points and alpha > 0");
    cudaStream_t st = c->stream;
    const int64_t np = le->npts;
    if(np > c->relax_cap) {
        if(c->d_relax) cudaFree(c->d_relax);
        c->d_relax = nullptr;
        c->relax_cap = 0;
        SPHGPU_CUDA(c, cudaMalloc(&c->d_relax, sizeof(double) * (size_t)(3 * np + 1)));
        c->relax_cap = np;
    }
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_relax, le->xi, sizeof(double) * np, cudaMemcpyHostToDevice, st));
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_relax + np, le->theta, sizeof(double) * np, cudaMemcpyHostToDevice, st));
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_relax + 2 * np, le->dtheta, sizeof(double) * np, cudaMemcpyHostToDevice, st));
    const unsigned g = grid_for(c->n, RBLK);
    if(first) k_relax_sound<<<g, RBLK, 0, st>>>(c->dp, c->s, c->n);
    int rc;
    if((rc = tree_make(c)) < 0) return rc;
    if((rc = pre_interaction(c)) < 0) return rc;
    if((rc = fluid_force(c)) < 0) return rc;
    if((rc = gravity(c, false)) < 0) return rc;
    k_relax_apply<<<g, RBLK, 0, st>>>(c->dp, c->s, c->n, c->d_relax, np, le->xi_1, le->alpha_scaling, le->K);
    if((rc = timestep(c)) < 0) return rc;
    k_relax_move<<<g, RBLK, 0, st>>>(c->dp, c->s, c->n, c->d_dt, c->d_relax + 3 * np);
    SPHGPU_LAUNCH_CHECK(c, "relax_step");
    double d = 0.0;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&d, c->d_relax + 3 * np, sizeof(double), cudaMemcpyDeviceToHost, st));
    SPHGPU_CUDA(c, cudaStreamSynchronize(st));
    stage_flush(c);
    if(dt_relax) *dt_relax = d;
    return SPHGPU_OK;
}
