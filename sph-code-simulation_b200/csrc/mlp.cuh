// mlp.cuh — learned initial guess for the GSPH iterative Riemann solver.
//
// No reference counterpart: the reference's iterative solver starts Newton
// from a PVRS-like linear guess (src/gsph/g_fluid_force.cpp:244-246).  The
// network maps the pair's left/right states to log(p_star / p_L):
//   x = (log(rho_R/rho_L), log(p_R/p_L), (u_R-u_L)/c_L, c_R/c_L, gamma)
//   3 hidden layers x 64, SiLU; BF16 weights, FP32 accumulation.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

struct sphgpu_ctx;

namespace sphgpu {

constexpr int MLP_IN = 5;
constexpr int MLP_INP = 16;   // input padded to one k-step of m16n8k16
constexpr int MLP_H = 64;
// parameter layout (FP32 master copy and the device image):
//   W0 [64][5], b0 [64], W1 [64][64], b1 [64], W2 [64][64], b2 [64], W3 [64], b3 [1]
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + 2 * (MLP_H * MLP_H + MLP_H) + MLP_H + 1;

// Device image used by inference: BF16 weights (W0 padded to 16 inputs),
// FP32 biases and input normalisation.
struct MlpDev {
    const __nv_bfloat16* w;   // W0p [64][16], W1 [64][64], W2 [64][64], W3 [64]
    const float* b;           // b0 [64], b1 [64], b2 [64], b3 [1]
};

MlpDev mlp_device(sphgpu_ctx* c);

// Features of a Riemann problem (left = j side, right = i side).
__device__ __forceinline__ void mlp_features(const double* L, const double* R, double gamma, float* x)
{
    const double cl = sqrt(gamma * L[2] / L[1]);
    const double cr = sqrt(gamma * R[2] / R[1]);
    x[0] = (float)log(R[1] / L[1]);
    x[1] = (float)log(R[2] / L[2]);
    x[2] = (float)((R[0] - L[0]) / cl);
    x[3] = (float)(cr / cl);
    x[4] = (float)gamma;
}

__device__ __forceinline__ float silu(float v) { return v / (1.0f + __expf(-v)); }

// Scalar (per-thread) forward pass; returns the guessed p_star (> 0) or -1
// when the states are not positive.
__device__ __forceinline__ double mlp_guess(const MlpDev& m, const double* L, const double* R, double gamma)
{
    if(!(L[1] > 0.0 && R[1] > 0.0 && L[2] > 0.0 && R[2] > 0.0)) return -1.0;
    float x[MLP_IN];
    mlp_features(L, R, gamma, x);
    float h0[MLP_H], h1[MLP_H];
    for(int o = 0; o < MLP_H; ++o) {
        float a = m.b[o];
        for(int k = 0; k < MLP_IN; ++k) a += __bfloat162float(m.w[o * MLP_INP + k]) * x[k];
        h0[o] = silu(a);
    }
    const __nv_bfloat16* w1 = m.w + MLP_H * MLP_INP;
    for(int o = 0; o < MLP_H; ++o) {
        float a = m.b[MLP_H + o];
        for(int k = 0; k < MLP_H; ++k) a += __bfloat162float(w1[o * MLP_H + k]) * h0[k];
        h1[o] = silu(a);
    }
    const __nv_bfloat16* w2 = w1 + MLP_H * MLP_H;
    for(int o = 0; o < MLP_H; ++o) {
        float a = m.b[2 * MLP_H + o];
        for(int k = 0; k < MLP_H; ++k) a += __bfloat162float(w2[o * MLP_H + k]) * h1[k];
        h0[o] = silu(a);
    }
    const __nv_bfloat16* w3 = w2 + MLP_H * MLP_H;
    float y = m.b[3 * MLP_H];
    for(int k = 0; k < MLP_H; ++k) y += __bfloat162float(w3[k]) * h0[k];
    return L[2] * exp((double)y);
}

}  // namespace sphgpu
