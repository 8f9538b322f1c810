// mlp.cuh — learned initial guess for the GSPH iterative Riemann solver.
//
// No reference counterpart: the reference's iterative solver starts Newton
// from a linearised guess (src/gsph/g_fluid_force.cpp:244-246).  The network
// maps a pair's left/right states to y = log(p_star / p_L):
//   features x = (log(rho_R/rho_L), log(p_R/p_L), (u_R-u_L)/c_L, c_R/c_L, gamma)
//   3 hidden layers x 64, SiLU; BF16 weights, FP32 accumulation.
// Inputs are scaled by fixed constants before the first layer (x0/7, x1/9,
// x2/5, min(x3, 64)/8, (gamma - 1.5) * 4) so every input is O(1).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

struct sphgpu_ctx;

namespace sphgpu {

constexpr int MLP_IN = 5;
constexpr int MLP_INP = 16;   // input padded to one k-step of m16n8k16
constexpr int MLP_H = 64;
// FP32 master parameter layout:
//   W0 [64][5], b0 [64], W1 [64][64], b1 [64], W2 [64][64], b2 [64], w3 [64], b3 [1]
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + 2 * (MLP_H * MLP_H + MLP_H) + MLP_H + 1;
constexpr int OFF_W0 = 0;
constexpr int OFF_B0 = OFF_W0 + MLP_H * MLP_IN;
constexpr int OFF_W1 = OFF_B0 + MLP_H;
constexpr int OFF_B1 = OFF_W1 + MLP_H * MLP_H;
constexpr int OFF_W2 = OFF_B1 + MLP_H;
constexpr int OFF_B2 = OFF_W2 + MLP_H * MLP_H;
constexpr int OFF_W3 = OFF_B2 + MLP_H;
constexpr int OFF_B3 = OFF_W3 + MLP_H;

// Device image (one allocation): BF16 W0p [64][16], W1 [64][64], W2 [64][64],
// W1^T, W2^T (backward), then FP32 w3 [64], b0, b1, b2 [64], b3.
constexpr int IMG_W0 = 0;
constexpr int IMG_W1 = IMG_W0 + MLP_H * MLP_INP;
constexpr int IMG_W2 = IMG_W1 + MLP_H * MLP_H;
constexpr int IMG_W1T = IMG_W2 + MLP_H * MLP_H;
constexpr int IMG_W2T = IMG_W1T + MLP_H * MLP_H;
constexpr int IMG_BF16 = IMG_W2T + MLP_H * MLP_H;              // bf16 elements
constexpr int IMG_F32_OFFSET = ((IMG_BF16 * 2 + 255) / 256) * 256; // bytes
constexpr int IMGF_W3 = 0, IMGF_B0 = 64, IMGF_B1 = 128, IMGF_B2 = 192, IMGF_B3 = 256;
constexpr int IMG_F32 = 260;
constexpr size_t IMG_BYTES = IMG_F32_OFFSET + IMG_F32 * 4;

struct MlpDev {
    const __nv_bfloat16* w;   // bf16 block of the image
    const float* f;           // fp32 block of the image
};

MlpDev mlp_device(sphgpu_ctx* c);

// Scaled features of a Riemann problem (left = j side, right = i side,
// state = (u, rho, p, c)); writes MLP_INP bf16 values (zero padded).
__device__ __forceinline__ void mlp_features(const double* L, const double* R, double gamma, float* x)
{
    const double cl = sqrt(gamma * L[2] / L[1]);
    const double cr = sqrt(gamma * R[2] / R[1]);
    x[0] = (float)(log(R[1] / L[1]) * (1.0 / 7.0));
    x[1] = (float)(log(R[2] / L[2]) * (1.0 / 9.0));
    x[2] = (float)((R[0] - L[0]) / cl * 0.2);
    x[3] = (float)(fmin(cr / cl, 64.0) * 0.125);
    x[4] = (float)((gamma - 1.5) * 4.0);
}

// Buffers of the learned path.  The force pass appends a row per pair whose
// linearised start the screen rejects (features: 8 bf16, 5 used; key: the pair
// slot i*cap + k), up to rcap rows; the network writes y[row] = log(p_star /
// p_L); after a sort by key, dstart/dcount give each particle's deferred rows,
// which the completion pass finishes in key order.
struct MlpPairs {
    uint4* feat;
    uint64_t* keys;
    unsigned long long* rows;
    long long rcap;
    const float* y;
    const uint64_t* skeys;    // sorted keys
    const uint32_t* svals;    // row of each sorted key
    const int* dstart;
    const int* dcount;
};

// Sampled pair states written by the plain solver (training data): records
// of 8 doubles (u_L, rho_L, p_L, u_R, rho_R, p_R, gamma, p_star).
struct Harvest {
    double* out;
    unsigned long long* count;
    long long cap;
    unsigned mod;     // keep a pair when hash(i, k) % mod == 0; 0 = off
    unsigned salt;
};
// Launchers (mlp.cu).
int mlp_infer_rows(sphgpu_ctx* c, const uint4* feat, float* y, long long rows);
int mlp_predict_states(sphgpu_ctx* c, const double* d_states, long long n, float* d_y);

__device__ __forceinline__ unsigned pack_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&v);
}

}  // namespace sphgpu
