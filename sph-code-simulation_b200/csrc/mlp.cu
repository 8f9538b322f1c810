// mlp.cu — parameters of the learned Riemann initial guess.
//
// FP32 master parameters (layout in mlp.cuh) are converted into the device
// inference image: BF16 weights (W0 zero-padded from 5 to 16 inputs so a
// layer is whole 16-wide k-steps) and FP32 biases.
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "context.cuh"
#include "mlp.cuh"

namespace sphgpu {

namespace {

constexpr size_t W_ELEMS = (size_t)MLP_H * MLP_INP + 2 * (size_t)MLP_H * MLP_H + MLP_H;
constexpr size_t B_OFFSET = (W_ELEMS * sizeof(__nv_bfloat16) + 255) / 256 * 256;
constexpr size_t B_ELEMS = 3 * MLP_H + 1;

}  // namespace

MlpDev mlp_device(sphgpu_ctx* c)
{
    MlpDev m{};
    if(!c->d_mlp) return m;
    m.w = static_cast<const __nv_bfloat16*>(c->d_mlp);
    m.b = reinterpret_cast<const float*>(static_cast<const char*>(c->d_mlp) + B_OFFSET);
    return m;
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int64_t sphgpu_mlp_param_count(void) { return MLP_NPARAM; }

int sphgpu_mlp_set_params(sphgpu_ctx* c, const float* params)
{
    if(!c || !params) return SPHGPU_ERR_ARG;
    c->mlp_master.assign(params, params + MLP_NPARAM);
    std::vector<__nv_bfloat16> w(W_ELEMS, __float2bfloat16(0.0f));
    std::vector<float> b(B_ELEMS, 0.0f);
    const float* p = params;
    for(int o = 0; o < MLP_H; ++o) {
        for(int k = 0; k < MLP_IN; ++k) w[(size_t)o * MLP_INP + k] = __float2bfloat16(p[o * MLP_IN + k]);
    }
    p += MLP_H * MLP_IN;
    for(int o = 0; o < MLP_H; ++o) b[o] = p[o];
    p += MLP_H;
    size_t wo = (size_t)MLP_H * MLP_INP;
    for(int l = 0; l < 2; ++l) {
        for(int k = 0; k < MLP_H * MLP_H; ++k) w[wo + k] = __float2bfloat16(p[k]);
        wo += (size_t)MLP_H * MLP_H;
        p += MLP_H * MLP_H;
        for(int o = 0; o < MLP_H; ++o) b[(size_t)(l + 1) * MLP_H + o] = p[o];
        p += MLP_H;
    }
    for(int k = 0; k < MLP_H; ++k) w[wo + k] = __float2bfloat16(p[k]);
    p += MLP_H;
    b[3 * MLP_H] = p[0];
    if(!c->d_mlp) {
        SPHGPU_CUDA(c, cudaMalloc(&c->d_mlp, B_OFFSET + B_ELEMS * sizeof(float)));
    }
    SPHGPU_CUDA(c, cudaMemcpy(c->d_mlp, w.data(), W_ELEMS * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    SPHGPU_CUDA(c, cudaMemcpy(static_cast<char*>(c->d_mlp) + B_OFFSET, b.data(), B_ELEMS * sizeof(float),
                              cudaMemcpyHostToDevice));
    c->have_mlp = true;
    return SPHGPU_OK;
}

int sphgpu_mlp_get_params(sphgpu_ctx* c, float* params)
{
    if(!c || !params) return SPHGPU_ERR_ARG;
    if(!c->have_mlp) return fail(c, SPHGPU_ERR_NO_MLP, "no MLP parameters loaded");
    std::memcpy(params, c->mlp_master.data(), sizeof(float) * MLP_NPARAM);
    return SPHGPU_OK;
}

}  // extern "C"
