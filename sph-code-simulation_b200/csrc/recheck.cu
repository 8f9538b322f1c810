// recheck.cu — the mixed form's FP64 re-evaluation.
//
// No counterpart in the reference.  The FP32 pair and gravity terms of the
// mixed form each carry a rounding error of a few units of 2^-24 of their own
// size; where they cancel (a pressure-balanced bulk, the centre of a
// self-gravitating sphere, a uniform state ahead of a shock) the summed
// acceleration keeps that absolute error while its own magnitude is small.
// FluidForce and GravityForce sum |term| beside the terms (accabs, per
// particle); after GravityForce every particle with
//     KAPPA * 2^-24 * accabs > mixed_acc_tol * (|a_x| + |a_y| + |a_z|)
// is listed (in index order) and its FluidForce and GravityForce are evaluated
// again in FP64 (the plain form's kernels on the same lists and tree), so its
// acceleration and du/dt are the FP64 form's.  KAPPA = 8 bounds the few
// roundings of one FP32 pair term and the FP32 partial sums of the gravity
// walk (checked against the FP64 form in tests/test_gpu_mixed.py).
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr double KAPPA = 8.0;
constexpr double EPS32 = 5.9604644775390625e-08;  // 2^-24

__global__ void k_recheck_flag(const double4* __restrict__ acc, const float* __restrict__ accabs, int n, double lim,
                               int* __restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const double4 a = acc[i];
    const double a1 = fabs(a.x) + fabs(a.y) + fabs(a.z);
    flag[i] = ((double)accabs[i] * lim > a1) ? 1 : 0;
}

__global__ void k_recheck_compact(const int* __restrict__ flag, const int* __restrict__ pos, int n,
                                  int* __restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n && flag[i]) idx[pos[i]] = i;
}

}  // namespace

int ensure_recheck(sphgpu_ctx* c)
{
    if(c->prm.precision != SPHGPU_MIXED) return SPHGPU_OK;
    if(c->recheck_n == c->n && c->d_recheck) return SPHGPU_OK;
    if(c->d_recheck) {
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        SPHGPU_CUDA(c, cudaFree(c->d_recheck));
        c->d_recheck = nullptr;
    }
    const size_t n = (size_t)c->n;
    // accabs (float), flag, pos, idx (int) and the count, 256-byte aligned pieces
    const size_t piece = (n * 4 + 255) / 256 * 256;
    SPHGPU_CUDA(c, cudaMalloc(&c->d_recheck, 4 * piece + 256));
    char* b = static_cast<char*>(c->d_recheck);
    c->d_accabs = reinterpret_cast<float*>(b);
    c->d_rflag = reinterpret_cast<int*>(b + piece);
    c->d_rpos = reinterpret_cast<int*>(b + 2 * piece);
    c->d_ridx = reinterpret_cast<int*>(b + 3 * piece);
    c->d_rcount = reinterpret_cast<int*>(b + 4 * piece);
    c->recheck_n = c->n;
    return SPHGPU_OK;
}

int mixed_recheck(sphgpu_ctx* c)
{
    if(c->prm.precision != SPHGPU_MIXED || !(c->prm.mixed_acc_tol > 0.0) || !c->accabs_valid) return SPHGPU_OK;
    c->accabs_valid = false;
    stage_begin(c, SPHGPU_T_RECHECK);
    const int n = c->n;
    const double lim = KAPPA * EPS32 / c->prm.mixed_acc_tol;
    k_recheck_flag<<<grid_for(n, 256), 256, 0, c->stream>>>(c->s.acc, c->d_accabs, n, lim, c->d_rflag);
    int launches = 2 + exclusive_scan(c->d_rflag, c->d_rpos, n, c->d_rcount, c->scan, c->stream);
    k_recheck_compact<<<grid_for(n, 256), 256, 0, c->stream>>>(c->d_rflag, c->d_rpos, n, c->d_ridx);
    SPHGPU_LAUNCH_CHECK(c, "mixed re-evaluation list");
    int nsub = 0;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&nsub, c->d_rcount, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if(nsub > 0) {
        int rc = fluid_force_subset64(c, c->d_ridx, nsub);
        if(rc < 0) return rc;
        rc = gravity_subset64(c, c->d_ridx, nsub);
        if(rc < 0) return rc;
        launches += c->prm.use_gravity ? 2 : 1;
    }
    c->mixed_rechecks += nsub;
    stage_end(c, SPHGPU_T_RECHECK, launches);
    return SPHGPU_OK;
}

}  // namespace sphgpu
