// noalloc.cu — TimeStep::calculation for callers that cannot allocate.
//
// sphgpu_timestep computes dt inside a context, whose reduction scratch the
// context allocated with cudaMalloc.  Some callers cannot allocate device
// memory at the point where they need dt: a host solver that owns the whole
// device memory budget through its own pool and forbids further cudaMalloc,
// or a caller that must not pay the device-wide synchronisation a
// cudaMalloc / cudaFree can imply.  sphgpu_timestep_noalloc serves them: the
// caller passes device arrays for the inputs and a device double for the
// result, and the per-block partial minima live in a fixed file-scope
// __device__ array instead of context memory.
//
// The array holds SPHGPU_NOALLOC_MAX_BLOCKS doubles (32 KiB); every GPU that
// loads this library keeps it until the process exits.  Each block covers
// SPHGPU_NOALLOC_TILE particles, so n is limited to
// SPHGPU_NOALLOC_MAX_PARTICLES; larger n is rejected with SPHGPU_ERR_ARG.
// Every call overwrites exactly the slots it reads, so nothing needs clearing
// between calls; calls that overlap on the GPU (different streams, or several
// host threads) share the array and race.
//
// Host code must not hand the array's name to a kernel: on the host it is
// only a stand-in.  The device address is looked up once per device with
// cudaGetSymbolAddress while that device is current; the first call on a
// device does this lookup, so that first call should come before any stream
// capture the caller starts.
#include <cfloat>
#include <mutex>
#include <cuda_runtime.h>

#include "sphgpu.h"

namespace {

constexpr int NA_BLOCK = 256;
constexpr int NA_ITEMS = 4;
constexpr int NA_TILE = NA_BLOCK * NA_ITEMS;   // = SPHGPU_NOALLOC_TILE
static_assert(NA_TILE == SPHGPU_NOALLOC_TILE, "tile size mismatch");

static __device__ __align__(256) double g_dt_partial[SPHGPU_NOALLOC_MAX_BLOCKS];

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
double* g_partial_ptr[MAX_DEVICES] = {nullptr};

// Minimum over one tile of cfl_force * sqrt(sml / |acc|) for |acc| > 0
// (src/timestep.cpp:24-32); DBL_MAX when the tile has no accelerated particle.
__global__ void __launch_bounds__(NA_BLOCK) k_na_dt_partial(const double* __restrict__ acc_xyz,
                                                            const double* __restrict__ sml, long long n,
                                                            double cfl_force, double* __restrict__ part)
{
    __shared__ double sm[NA_BLOCK / 32];
    double m = DBL_MAX;
    const long long base = (long long)blockIdx.x * NA_TILE;
#pragma unroll
    for(int k = 0; k < NA_ITEMS; ++k) {
        const long long i = base + (long long)k * NA_BLOCK + threadIdx.x;
        if(i < n) {
            const double ax = acc_xyz[3 * i], ay = acc_xyz[3 * i + 1], az = acc_xyz[3 * i + 2];
            const double aa = sqrt(ax * ax + ay * ay + az * az);
            if(aa > 0.0) {
                const double d = cfl_force * sqrt(sml[i] / aa);
                if(d < m) m = d;
            }
        }
    }
    for(int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, m, o);
        m = u < m ? u : m;
    }
    if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if(threadIdx.x == 0) {
        for(int w = 1; w < NA_BLOCK / 32; ++w) m = fmin(m, sm[w]);
        part[blockIdx.x] = fmin(m, sm[0]);
    }
}

// dt = min(cfl_sound * h_per_v_sig, min over tiles) (src/timestep.cpp:34-37)
__global__ void __launch_bounds__(NA_BLOCK) k_na_dt_final(const double* __restrict__ part, int nb, double hvs,
                                                          double cfl_sound, double* __restrict__ dt_out)
{
    __shared__ double sm[NA_BLOCK / 32];
    double m = DBL_MAX;
    for(int b = threadIdx.x; b < nb; b += NA_BLOCK) m = fmin(m, part[b]);
    for(int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, m, o);
        m = u < m ? u : m;
    }
    if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if(threadIdx.x == 0) {
        for(int w = 1; w < NA_BLOCK / 32; ++w) m = fmin(m, sm[w]);
        m = fmin(m, sm[0]);
        const double ds = cfl_sound * hvs;
        *dt_out = m < ds ? m : ds;  // std::min(dt_sound, dt_force)
    }
}

// Device address of g_dt_partial on the current device (looked up once).
int partial_address(double** out)
{
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return SPHGPU_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    if(!g_partial_ptr[dev]) {
        void* p = nullptr;
        if(cudaGetSymbolAddress(&p, g_dt_partial) != cudaSuccess || !p) return SPHGPU_ERR_CUDA;
        g_partial_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_partial_ptr[dev];
    return SPHGPU_OK;
}

}  // namespace

extern "C" int sphgpu_timestep_noalloc(const double* acc_xyz, const double* sml, int64_t n, double h_per_v_sig,
                                       double cfl_sound, double cfl_force, double* dt_out, void* stream)
{
    if(!acc_xyz || !sml || !dt_out || n <= 0) return SPHGPU_ERR_ARG;
    if(n > (int64_t)SPHGPU_NOALLOC_MAX_PARTICLES) return SPHGPU_ERR_ARG;
    double* part = nullptr;
    const int rc = partial_address(&part);
    if(rc != SPHGPU_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = (int)((n + NA_TILE - 1) / NA_TILE);
    k_na_dt_partial<<<nb, NA_BLOCK, 0, st>>>(acc_xyz, sml, (long long)n, cfl_force, part);
    k_na_dt_final<<<1, NA_BLOCK, 0, st>>>(part, nb, h_per_v_sig, cfl_sound, dt_out);
    return cudaGetLastError() == cudaSuccess ? SPHGPU_OK : SPHGPU_ERR_CUDA;
}
