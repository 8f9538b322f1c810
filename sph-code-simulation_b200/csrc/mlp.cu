// mlp.cu — tensor-core inference and training of the learned Riemann guess.
//
// Network (mlp.cuh): 5 scaled inputs (padded to 16) -> 64 -> 64 -> 64 -> 1,
// SiLU, BF16 weights / activations, FP32 accumulation.  Every matrix product
// is a warp-level mma.sync.m16n8k16 (bf16 x bf16 -> f32) on a 16-row tile:
//   * a layer's f32 accumulator fragments (two adjacent 8-column n-tiles) are
//     exactly the bf16 A-operand fragment of the next layer's k-tile, so the
//     three hidden layers stay in registers;
//   * training computes weight gradients dW = dZ^T A_prev on the same 16-row
//     tile: movmatrix.trans turns the accumulator / operand fragments into the
//     transposed operands, and the 16-row partial products are accumulated in
//     shared memory (f32 atomics), then once per block into global memory.
// Training keeps FP32 master parameters and Adam moments; the BF16 image the
// kernels read is rebuilt after every update.
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "context.cuh"
#include "mlp.cuh"

namespace sphgpu {

namespace {

constexpr int LDW0 = 24;  // padded smem row lengths (bf16) for conflict-free fragment loads
constexpr int LDW = 72;

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned trans8x8(unsigned a)
{
    unsigned d;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(d) : "r"(a));
    return d;
}

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_(float z) { return z * sigmoidf_(z); }
__device__ __forceinline__ float dsilu_(float z)
{
    const float s = sigmoidf_(z);
    return s * (1.0f + z * (1.0f - s));
}

// Shared-memory copy of the network (inference and training forward).
struct SmemNet {
    __nv_bfloat16 w0[MLP_H * LDW0];
    __nv_bfloat16 w1[MLP_H * LDW];
    __nv_bfloat16 w2[MLP_H * LDW];
    float w3[MLP_H];
    float b0[MLP_H], b1[MLP_H], b2[MLP_H];
    float b3;
};

__device__ void load_net(SmemNet& s, const MlpDev& m)
{
    for(int k = threadIdx.x; k < MLP_H * MLP_INP; k += blockDim.x) {
        s.w0[(k / MLP_INP) * LDW0 + (k % MLP_INP)] = m.w[IMG_W0 + k];
    }
    for(int k = threadIdx.x; k < MLP_H * MLP_H; k += blockDim.x) {
        s.w1[(k / MLP_H) * LDW + (k % MLP_H)] = m.w[IMG_W1 + k];
        s.w2[(k / MLP_H) * LDW + (k % MLP_H)] = m.w[IMG_W2 + k];
    }
    for(int k = threadIdx.x; k < MLP_H; k += blockDim.x) {
        s.w3[k] = m.f[IMGF_W3 + k];
        s.b0[k] = m.f[IMGF_B0 + k];
        s.b1[k] = m.f[IMGF_B1 + k];
        s.b2[k] = m.f[IMGF_B2 + k];
    }
    if(threadIdx.x == 0) s.b3 = m.f[IMGF_B3];
}

// B fragment (k = 16 kk + {2t, 2t+1, 2t+8, 2t+9}, n = 8 j + g) of W^T for a
// row-major W[out][in] in smem with row length ld: element (k, n) = W[n][k].
__device__ __forceinline__ void bfrag(const __nv_bfloat16* w, int ld, int j, int kk, int g, int t, unsigned& b0,
                                      unsigned& b1)
{
    const __nv_bfloat16* row = w + (8 * j + g) * ld + 16 * kk + 2 * t;
    b0 = *reinterpret_cast<const unsigned*>(row);
    b1 = *reinterpret_cast<const unsigned*>(row + 8);
}

// Forward of one 16-row tile.  a0x[4]: input fragment.  Returns pre-activations
// z[layer][ntile][4] when Z is non-null (training) and y for rows g, g+8.
template <bool KEEP>
__device__ __forceinline__ void forward_tile(const SmemNet& s, const unsigned (&ax)[4], int g, int t,
                                             float (*Z)[8][4], unsigned (*A)[4][4], float& y_lo, float& y_hi,
                                             float (&a3)[8][4])
{
    float c[8][4];
    // layer 0: K = 16
#pragma unroll
    for(int j = 0; j < 8; ++j) {
        c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
        unsigned b0, b1;
        bfrag(s.w0, LDW0, j, 0, g, t, b0, b1);
        mma16816(c[j], ax[0], ax[1], ax[2], ax[3], b0, b1);
    }
    unsigned act[4][4];
#pragma unroll
    for(int layer = 0; layer < 3; ++layer) {
        const float* bias = layer == 0 ? s.b0 : (layer == 1 ? s.b1 : s.b2);
        float a[8][4];
#pragma unroll
        for(int j = 0; j < 8; ++j) {
            const float bl = bias[8 * j + 2 * t], bh = bias[8 * j + 2 * t + 1];
            c[j][0] += bl;
            c[j][1] += bh;
            c[j][2] += bl;
            c[j][3] += bh;
#pragma unroll
            for(int e = 0; e < 4; ++e) {
                if(KEEP) Z[layer][j][e] = c[j][e];
                a[j][e] = silu_(c[j][e]);
            }
        }
        if(layer == 2) {
#pragma unroll
            for(int j = 0; j < 8; ++j) {
#pragma unroll
                for(int e = 0; e < 4; ++e) a3[j][e] = a[j][e];
            }
            break;
        }
#pragma unroll
        for(int kk = 0; kk < 4; ++kk) {
            act[kk][0] = pack_bf16(a[2 * kk][0], a[2 * kk][1]);
            act[kk][1] = pack_bf16(a[2 * kk][2], a[2 * kk][3]);
            act[kk][2] = pack_bf16(a[2 * kk + 1][0], a[2 * kk + 1][1]);
            act[kk][3] = pack_bf16(a[2 * kk + 1][2], a[2 * kk + 1][3]);
            if(KEEP) {
#pragma unroll
                for(int e = 0; e < 4; ++e) A[layer][kk][e] = act[kk][e];
            }
        }
        const __nv_bfloat16* w = layer == 0 ? s.w1 : s.w2;
#pragma unroll
        for(int j = 0; j < 8; ++j) {
            c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
            for(int kk = 0; kk < 4; ++kk) {
                unsigned b0, b1;
                bfrag(w, LDW, j, kk, g, t, b0, b1);
                mma16816(c[j], act[kk][0], act[kk][1], act[kk][2], act[kk][3], b0, b1);
            }
        }
    }
    // output: y = a3 . w3 + b3, reduced over the 4 lanes of a row group
    float lo = 0.f, hi = 0.f;
#pragma unroll
    for(int j = 0; j < 8; ++j) {
        const float wl = s.w3[8 * j + 2 * t], wh = s.w3[8 * j + 2 * t + 1];
        lo += a3[j][0] * wl + a3[j][1] * wh;
        hi += a3[j][2] * wl + a3[j][3] * wh;
    }
    lo += __shfl_xor_sync(FULL_MASK, lo, 1);
    lo += __shfl_xor_sync(FULL_MASK, lo, 2);
    hi += __shfl_xor_sync(FULL_MASK, hi, 1);
    hi += __shfl_xor_sync(FULL_MASK, hi, 2);
    y_lo = lo + s.b3;
    y_hi = hi + s.b3;
}

// input fragment of rows r0 + g, r0 + g + 8 from 8-bf16 feature rows
__device__ __forceinline__ void load_input(const uint4* __restrict__ feat, long long r_lo, long long r_hi, bool v_lo,
                                           bool v_hi, int t, unsigned (&ax)[4])
{
    const unsigned* lo = reinterpret_cast<const unsigned*>(feat + r_lo);
    const unsigned* hi = reinterpret_cast<const unsigned*>(feat + r_hi);
    ax[0] = v_lo ? lo[t] : 0u;   // cols 2t, 2t+1 (features 0..7)
    ax[1] = v_hi ? hi[t] : 0u;
    ax[2] = 0u;                  // cols 8..15: padding
    ax[3] = 0u;
}

constexpr int IBLK = 128;

// y[row] for feature rows (8 bf16 per row, 5 used).
__global__ void __launch_bounds__(IBLK) k_mlp_infer(MlpDev m, const uint4* __restrict__ feat, float* __restrict__ y,
                                                    long long rows)
{
    __shared__ SmemNet s;
    load_net(s, m);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long warp = ((long long)blockIdx.x * IBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * IBLK) >> 5;
    const long long tiles = (rows + 15) / 16;
    for(long long tile = warp; tile < tiles; tile += nwarps) {
        const long long r0 = tile * 16;
        const long long rl = r0 + g, rh = r0 + g + 8;
        unsigned ax[4];
        load_input(feat, rl < rows ? rl : 0, rh < rows ? rh : 0, rl < rows, rh < rows, t, ax);
        float ylo, yhi, a3[8][4];
        forward_tile<false>(s, ax, g, t, nullptr, nullptr, ylo, yhi, a3);
        if(t == 0) {
            if(rl < rows) y[rl] = ylo;
            if(rh < rows) y[rh] = yhi;
        }
    }
}

// --------------------------------------------------------------- training
struct SmemGrad {
    float w0[MLP_H * MLP_IN];
    float b0[MLP_H];
    float w1[MLP_H * MLP_H];
    float b1[MLP_H];
    float w2[MLP_H * MLP_H];
    float b2[MLP_H];
    float w3[MLP_H];
    float b3;
    float loss;
};

constexpr int TBLK = 128;
constexpr size_t align16(size_t x) { return (x + 15) / 16 * 16; }
constexpr size_t TRAIN_OFF_W1T = align16(sizeof(SmemNet));
constexpr size_t TRAIN_OFF_W2T = TRAIN_OFF_W1T + align16(sizeof(__nv_bfloat16) * MLP_H * LDW);
constexpr size_t TRAIN_OFF_GRAD = TRAIN_OFF_W2T + align16(sizeof(__nv_bfloat16) * MLP_H * LDW);
constexpr size_t TRAIN_SMEM = TRAIN_OFF_GRAD + align16(sizeof(SmemGrad));

// B fragment of W (not transposed) for dA = dZ W: element (k = out, n = in) =
// W[k][n] = WT[n][k] with WT row-major in smem.
__device__ __forceinline__ void bfragT(const __nv_bfloat16* wt, int j, int kk, int g, int t, unsigned& b0,
                                       unsigned& b1)
{
    const __nv_bfloat16* row = wt + (8 * j + g) * LDW + 16 * kk + 2 * t;
    b0 = *reinterpret_cast<const unsigned*>(row);
    b1 = *reinterpret_cast<const unsigned*>(row + 8);
}

// Accumulate dW[o][i] += sum_r dZ[r][o] Aprev[r][i] for one 16-row tile.
// dzA: dZ as bf16 A-fragments (4 k-tiles over o); ap: Aprev as A-fragments
// (k-tiles over i, nk of them); out: smem f32 [64][nin].
__device__ __forceinline__ void weight_grad(const unsigned (&dzA)[4][4], const unsigned (*ap)[4], int nk, int nin,
                                            float* out, int g, int t)
{
#pragma unroll
    for(int p = 0; p < 4; ++p) {        // o-tile: o = 16p .. 16p+15
        // A operand rows o, k = rows r: transposes of the dZ sub-blocks
        const unsigned a0 = trans8x8(dzA[p][0]);   // rows 0-7,  o 16p..16p+7
        const unsigned a1 = trans8x8(dzA[p][2]);   // rows 0-7,  o 16p+8..
        const unsigned a2 = trans8x8(dzA[p][1]);   // rows 8-15, o 16p..
        const unsigned a3 = trans8x8(dzA[p][3]);   // rows 8-15, o 16p+8..
        for(int kk = 0; kk < nk; ++kk) {
            for(int h = 0; h < 2; ++h) {   // n-tile over inputs i = 16kk + 8h + (0..7)
                const unsigned b0 = trans8x8(ap[kk][h == 0 ? 0 : 2]);
                const unsigned b1 = trans8x8(ap[kk][h == 0 ? 1 : 3]);
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                mma16816(d, a0, a1, a2, a3, b0, b1);
                const int o = 16 * p + g, i = 16 * kk + 8 * h + 2 * t;
                if(i < nin) {
                    atomicAdd(&out[o * nin + i], d[0]);
                    atomicAdd(&out[(o + 8) * nin + i], d[2]);
                }
                if(i + 1 < nin) {
                    atomicAdd(&out[o * nin + i + 1], d[1]);
                    atomicAdd(&out[(o + 8) * nin + i + 1], d[3]);
                }
            }
        }
    }
}

// Column sums of a C-layout tile (bias gradients) into smem.
__device__ __forceinline__ void bias_grad(const float (&dz)[8][4], float* out, int g, int t)
{
#pragma unroll
    for(int j = 0; j < 8; ++j) {
        float s0 = dz[j][0] + dz[j][2], s1 = dz[j][1] + dz[j][3];
        for(int o = 4; o < 32; o <<= 1) {
            s0 += __shfl_xor_sync(FULL_MASK, s0, o);
            s1 += __shfl_xor_sync(FULL_MASK, s1, o);
        }
        if(g == 0) {
            atomicAdd(&out[8 * j + 2 * t], s0);
            atomicAdd(&out[8 * j + 2 * t + 1], s1);
        }
    }
}

// One training batch: rows r = perm(batch_base + k), k < bsize; loss = mean
// of (y - target)^2 over the batch.  Gradients are summed into grad (global).
__global__ void __launch_bounds__(TBLK) k_mlp_train(MlpDev m, const __nv_bfloat16* __restrict__ wt1,
                                                    const __nv_bfloat16* __restrict__ wt2,
                                                    const uint4* __restrict__ feat, const float* __restrict__ target,
                                                    long long nrows, long long batch_base, int bsize,
                                                    unsigned long long pa, unsigned long long pc,
                                                    float* __restrict__ grad, float* __restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemNet& s = *reinterpret_cast<SmemNet*>(smem_raw);
    __nv_bfloat16* s_w1t = reinterpret_cast<__nv_bfloat16*>(smem_raw + TRAIN_OFF_W1T);
    __nv_bfloat16* s_w2t = reinterpret_cast<__nv_bfloat16*>(smem_raw + TRAIN_OFF_W2T);
    SmemGrad& sg = *reinterpret_cast<SmemGrad*>(smem_raw + TRAIN_OFF_GRAD);
    load_net(s, m);
    for(int k = threadIdx.x; k < MLP_H * MLP_H; k += TBLK) {
        s_w1t[(k / MLP_H) * LDW + (k % MLP_H)] = wt1[k];
        s_w2t[(k / MLP_H) * LDW + (k % MLP_H)] = wt2[k];
    }
    float* sgf = reinterpret_cast<float*>(&sg);
    for(int k = threadIdx.x; k < (int)(sizeof(SmemGrad) / 4); k += TBLK) sgf[k] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warp = (blockIdx.x * TBLK + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * TBLK) >> 5;
    const float inv_b = 1.0f / (float)bsize;
    const int tiles = (bsize + 15) / 16;
    for(int tile = warp; tile < tiles; tile += nwarps) {
        const int k_lo = tile * 16 + g, k_hi = k_lo + 8;
        const bool v_lo = k_lo < bsize, v_hi = k_hi < bsize;
        const long long r_lo = v_lo ? (long long)((pa * (unsigned long long)(batch_base + k_lo) + pc) % nrows) : 0;
        const long long r_hi = v_hi ? (long long)((pa * (unsigned long long)(batch_base + k_hi) + pc) % nrows) : 0;
        unsigned ax[4];
        load_input(feat, r_lo, r_hi, v_lo, v_hi, t, ax);
        float Z[3][8][4];
        unsigned A[2][4][4];
        float a3[8][4], ylo, yhi;
        forward_tile<true>(s, ax, g, t, Z, A, ylo, yhi, a3);
        const float elo = v_lo ? ylo - target[r_lo] : 0.f;
        const float ehi = v_hi ? yhi - target[r_hi] : 0.f;
        if(t == 0) {
            float l = elo * elo + ehi * ehi;
            for(int o = 4; o < 32; o <<= 1) l += __shfl_xor_sync(0x11111111u, l, o);
            if(g == 0) atomicAdd(&sg.loss, l * inv_b);
        }
        const float dlo = 2.f * elo * inv_b, dhi = 2.f * ehi * inv_b;
        // output layer: dw3, db3, dZ3
        float dz[8][4];
#pragma unroll
        for(int j = 0; j < 8; ++j) {
            float s0 = dlo * a3[j][0] + dhi * a3[j][2], s1 = dlo * a3[j][1] + dhi * a3[j][3];
            for(int o = 4; o < 32; o <<= 1) {
                s0 += __shfl_xor_sync(FULL_MASK, s0, o);
                s1 += __shfl_xor_sync(FULL_MASK, s1, o);
            }
            if(g == 0) {
                atomicAdd(&sg.w3[8 * j + 2 * t], s0);
                atomicAdd(&sg.w3[8 * j + 2 * t + 1], s1);
            }
            const float wl = s.w3[8 * j + 2 * t], wh = s.w3[8 * j + 2 * t + 1];
            dz[j][0] = dlo * wl * dsilu_(Z[2][j][0]);
            dz[j][1] = dlo * wh * dsilu_(Z[2][j][1]);
            dz[j][2] = dhi * wl * dsilu_(Z[2][j][2]);
            dz[j][3] = dhi * wh * dsilu_(Z[2][j][3]);
        }
        {
            float sb = dlo + dhi;
            for(int o = 4; o < 32; o <<= 1) sb += __shfl_xor_sync(FULL_MASK, sb, o);
            if(lane == 0) atomicAdd(&sg.b3, sb);
        }
        // hidden layers 2 .. 0
        for(int layer = 2; layer >= 0; --layer) {
            bias_grad(dz, layer == 2 ? sg.b2 : (layer == 1 ? sg.b1 : sg.b0), g, t);
            unsigned dzA[4][4];
#pragma unroll
            for(int kk = 0; kk < 4; ++kk) {
                dzA[kk][0] = pack_bf16(dz[2 * kk][0], dz[2 * kk][1]);
                dzA[kk][1] = pack_bf16(dz[2 * kk][2], dz[2 * kk][3]);
                dzA[kk][2] = pack_bf16(dz[2 * kk + 1][0], dz[2 * kk + 1][1]);
                dzA[kk][3] = pack_bf16(dz[2 * kk + 1][2], dz[2 * kk + 1][3]);
            }
            if(layer == 0) {
                const unsigned xin[1][4] = {{ax[0], ax[1], ax[2], ax[3]}};
                weight_grad(dzA, xin, 1, MLP_IN, sg.w0, g, t);
                break;
            }
            weight_grad(dzA, A[layer - 1], 4, MLP_H, layer == 2 ? sg.w2 : sg.w1, g, t);
            // dA_prev = dZ W, dZ_prev = dA_prev * silu'(Z_prev)
            const __nv_bfloat16* wt = layer == 2 ? s_w2t : s_w1t;
            float da[8][4];
#pragma unroll
            for(int j = 0; j < 8; ++j) {
                da[j][0] = da[j][1] = da[j][2] = da[j][3] = 0.f;
#pragma unroll
                for(int kk = 0; kk < 4; ++kk) {
                    unsigned b0, b1;
                    bfragT(wt, j, kk, g, t, b0, b1);
                    mma16816(da[j], dzA[kk][0], dzA[kk][1], dzA[kk][2], dzA[kk][3], b0, b1);
                }
#pragma unroll
                for(int e = 0; e < 4; ++e) dz[j][e] = da[j][e] * dsilu_(Z[layer - 1][j][e]);
            }
        }
    }
    __syncthreads();
    for(int k = threadIdx.x; k < MLP_NPARAM; k += TBLK) {
        // smem gradient layout equals the master parameter layout
        const float v = sgf[k];
        if(v != 0.f) atomicAdd(&grad[k], v);
    }
    if(threadIdx.x == 0) atomicAdd(loss, sg.loss);
}

// Adam update of the FP32 master parameters, then the BF16 image.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, int n, float lr, float b1, float b2, float c1, float c2, float eps)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= n) return;
    const float gk = grad[k];
    const float a = b1 * m1[k] + (1.f - b1) * gk;
    const float b = b2 * m2[k] + (1.f - b2) * gk * gk;
    m1[k] = a;
    m2[k] = b;
    p[k] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

__global__ void k_make_image(const float* __restrict__ p, __nv_bfloat16* __restrict__ w, float* __restrict__ f)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < MLP_H * MLP_INP + 4 * MLP_H * MLP_H + 4 * MLP_H + 1;
        k += gridDim.x * blockDim.x) {
        if(k < MLP_H * MLP_INP) {
            const int o = k / MLP_INP, i = k % MLP_INP;
            w[IMG_W0 + k] = __float2bfloat16(i < MLP_IN ? p[OFF_W0 + o * MLP_IN + i] : 0.f);
            continue;
        }
        int q = k - MLP_H * MLP_INP;
        if(q < 4 * MLP_H * MLP_H) {
            const int which = q / (MLP_H * MLP_H), e = q % (MLP_H * MLP_H);
            const int r = e / MLP_H, cidx = e % MLP_H;
            if(which == 0) w[IMG_W1 + e] = __float2bfloat16(p[OFF_W1 + e]);
            else if(which == 1) w[IMG_W2 + e] = __float2bfloat16(p[OFF_W2 + e]);
            else if(which == 2) w[IMG_W1T + e] = __float2bfloat16(p[OFF_W1 + cidx * MLP_H + r]);
            else w[IMG_W2T + e] = __float2bfloat16(p[OFF_W2 + cidx * MLP_H + r]);
            continue;
        }
        q -= 4 * MLP_H * MLP_H;
        if(q < MLP_H) f[IMGF_W3 + q] = p[OFF_W3 + q];
        else if(q < 2 * MLP_H) f[IMGF_B0 + q - MLP_H] = p[OFF_B0 + q - MLP_H];
        else if(q < 3 * MLP_H) f[IMGF_B1 + q - 2 * MLP_H] = p[OFF_B1 + q - 2 * MLP_H];
        else if(q < 4 * MLP_H) f[IMGF_B2 + q - 3 * MLP_H] = p[OFF_B2 + q - 3 * MLP_H];
        else f[IMGF_B3] = p[OFF_B3];
    }
}

// Features + targets of raw Riemann states (n x 7: uL rhoL pL uR rhoR pR gamma).
__global__ void k_state_features(const double* __restrict__ st, const double* __restrict__ pstar, long long n,
                                 uint4* __restrict__ feat, float* __restrict__ target)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= n) return;
    const double* s = st + 7 * r;
    const double gamma = s[6];
    const double L[4] = {s[0], s[1], s[2], sqrt(gamma * s[2] / s[1])};
    const double R[4] = {s[3], s[4], s[5], sqrt(gamma * s[5] / s[4])};
    float x[MLP_IN];
    mlp_features(L, R, gamma, x);
    uint4 v;
    v.x = pack_bf16(x[0], x[1]);
    v.y = pack_bf16(x[2], x[3]);
    v.z = pack_bf16(x[4], 0.f);
    v.w = 0u;
    feat[r] = v;
    if(target) target[r] = (float)log(pstar[r] / s[2]);
}

}  // namespace

MlpDev mlp_device(sphgpu_ctx* c)
{
    MlpDev m{};
    if(!c->d_mlp) return m;
    m.w = static_cast<const __nv_bfloat16*>(c->d_mlp);
    m.f = reinterpret_cast<const float*>(static_cast<const char*>(c->d_mlp) + IMG_F32_OFFSET);
    return m;
}

int mlp_infer_rows(sphgpu_ctx* c, const uint4* feat, float* y, long long rows)
{
    const long long tiles = (rows + 15) / 16;
    const long long blocks = std::min<long long>((tiles + (IBLK / 32) - 1) / (IBLK / 32), 148LL * 16);
    k_mlp_infer<<<(unsigned)std::max<long long>(blocks, 1), IBLK, 0, c->stream>>>(mlp_device(c), feat, y, rows);
    SPHGPU_LAUNCH_CHECK(c, "MLP inference");
    return SPHGPU_OK;
}

// y for device-resident states (n x 7); d_y has n floats.
int mlp_predict_states(sphgpu_ctx* c, const double* d_states, long long n, float* d_y)
{
    uint4* feat = nullptr;
    DevTemps tmp(c->stream);
    SPHGPU_CUDA(c, tmp.get(&feat, sizeof(uint4) * (size_t)n, false));
    k_state_features<<<grid_for(n, 256), 256, 0, c->stream>>>(d_states, nullptr, n, feat, nullptr);
    const long long tiles = (n + 15) / 16;
    const long long blocks = std::min<long long>((tiles + 3) / 4, 148LL * 16);
    k_mlp_infer<<<(unsigned)std::max<long long>(blocks, 1), IBLK, 0, c->stream>>>(mlp_device(c), feat, d_y, n);
    SPHGPU_LAUNCH_CHECK(c, "MLP predict");
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return SPHGPU_OK;
}

static int ensure_image(sphgpu_ctx* c)
{
    if(!c->d_mlp) SPHGPU_CUDA(c, cudaMalloc(&c->d_mlp, IMG_BYTES));
    return SPHGPU_OK;
}

static int upload_master(sphgpu_ctx* c)
{
    int rc = ensure_image(c);
    if(rc) return rc;
    if(!c->d_mlp_master) SPHGPU_CUDA(c, cudaMalloc(&c->d_mlp_master, sizeof(float) * 4 * MLP_NPARAM));
    SPHGPU_CUDA(c, cudaMemcpy(c->d_mlp_master, c->mlp_master.data(), sizeof(float) * MLP_NPARAM,
                              cudaMemcpyHostToDevice));
    k_make_image<<<64, 256, 0, c->stream>>>(c->d_mlp_master, static_cast<__nv_bfloat16*>(c->d_mlp),
                                            reinterpret_cast<float*>(static_cast<char*>(c->d_mlp) + IMG_F32_OFFSET));
    SPHGPU_LAUNCH_CHECK(c, "MLP image");
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_mlp = true;
    return SPHGPU_OK;
}

// device features/targets for host states, in buffers taken from `keep`
// (released with it by the caller's scope)
static int stage_states(sphgpu_ctx* c, DevTemps& keep, const double* states, const double* pstar, int64_t n,
                        uint4** feat, float** target)
{
    double *d_st = nullptr, *d_ps = nullptr;
    DevTemps tmp(c->stream);
    SPHGPU_CUDA(c, tmp.get(&d_st, sizeof(double) * 7 * (size_t)n, false));
    SPHGPU_CUDA(c, cudaMemcpyAsync(d_st, states, sizeof(double) * 7 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    if(pstar) {
        SPHGPU_CUDA(c, tmp.get(&d_ps, sizeof(double) * (size_t)n, false));
        SPHGPU_CUDA(c, cudaMemcpyAsync(d_ps, pstar, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    }
    SPHGPU_CUDA(c, keep.get(feat, sizeof(uint4) * (size_t)n, false));
    *target = nullptr;
    if(pstar) SPHGPU_CUDA(c, keep.get(target, sizeof(float) * (size_t)n, false));
    k_state_features<<<grid_for(n, 256), 256, 0, c->stream>>>(d_st, d_ps, n, *feat, *target);
    SPHGPU_LAUNCH_CHECK(c, "MLP features");
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return SPHGPU_OK;
}

}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

int64_t sphgpu_mlp_param_count(void) { return MLP_NPARAM; }

int sphgpu_mlp_set_params(sphgpu_ctx* c, const float* params)
{
    if(!c || !params) return SPHGPU_ERR_ARG;
    if(!c->stream) return fail(c, SPHGPU_ERR_CUDA, "context has no device");
    c->mlp_master.assign(params, params + MLP_NPARAM);
    return upload_master(c);
}

int sphgpu_mlp_get_params(sphgpu_ctx* c, float* params)
{
    if(!c || !params) return SPHGPU_ERR_ARG;
    if(!c->have_mlp) return fail(c, SPHGPU_ERR_NO_MLP, "no MLP parameters loaded");
    std::memcpy(params, c->mlp_master.data(), sizeof(float) * MLP_NPARAM);
    return SPHGPU_OK;
}

// Deterministic initialisation (uniform +-sqrt(6 / (fan_in + fan_out)), zero
// biases) from a 64-bit seed.
int sphgpu_mlp_init(sphgpu_ctx* c, uint64_t seed)
{
    if(!c) return SPHGPU_ERR_ARG;
    std::vector<float> p(MLP_NPARAM, 0.f);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
    auto uni = [&]() {
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        return (double)((x * 0x2545F4914F6CDD1Dull) >> 11) / 9007199254740992.0;
    };
    auto fill = [&](int off, int fan_in, int fan_out, int count) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for(int k = 0; k < count; ++k) p[off + k] = (float)((2.0 * uni() - 1.0) * a);
    };
    fill(OFF_W0, MLP_IN, MLP_H, MLP_H * MLP_IN);
    fill(OFF_W1, MLP_H, MLP_H, MLP_H * MLP_H);
    fill(OFF_W2, MLP_H, MLP_H, MLP_H * MLP_H);
    fill(OFF_W3, MLP_H, 1, MLP_H);
    return sphgpu_mlp_set_params(c, p.data());
}

// y = network output log(p_star / p_L) for raw states (n x 7).
int sphgpu_mlp_predict(sphgpu_ctx* c, const double* states, int64_t n, float* y)
{
    if(!c || !states || !y || n <= 0) return SPHGPU_ERR_ARG;
    if(!c->have_mlp) return fail(c, SPHGPU_ERR_NO_MLP, "no MLP parameters loaded");
    uint4* feat = nullptr;
    float* tgt = nullptr;
    DevTemps tmp(c->stream);
    int rc = stage_states(c, tmp, states, nullptr, n, &feat, &tgt);
    if(rc) return rc;
    float* d_y = nullptr;
    SPHGPU_CUDA(c, tmp.get(&d_y, sizeof(float) * (size_t)n, false));
    const long long tiles = (n + 15) / 16;
    const long long blocks = std::min<long long>((tiles + 3) / 4, 148LL * 16);
    k_mlp_infer<<<(unsigned)blocks, IBLK, 0, c->stream>>>(mlp_device(c), feat, d_y, n);
    SPHGPU_LAUNCH_CHECK(c, "MLP predict");
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));  // the context stream does not sync with cudaMemcpy
    SPHGPU_CUDA(c, cudaMemcpy(y, d_y, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    return SPHGPU_OK;
}

// Train on labelled states with Adam (mean squared error in log(p*/p_L)).
// loss_history[e] = mean batch loss of epoch e.  With epochs == 0 only the
// full-data gradient of the current parameters is written to grad_out (for
// gradient checks) and its loss to loss_history[0].
int sphgpu_mlp_train(sphgpu_ctx* c, const double* states, const double* pstar, int64_t n, int epochs, int batch,
                     float lr, uint64_t seed, float* loss_history, float* grad_out)
{
    if(!c || !states || !pstar || n <= 0 || batch <= 0 || epochs < 0) return SPHGPU_ERR_ARG;
    if(!c->have_mlp) {
        const int rc = sphgpu_mlp_init(c, seed);
        if(rc) return rc;
    }
    uint4* feat = nullptr;
    float* tgt = nullptr;
    DevTemps tmp(c->stream);
    int rc = stage_states(c, tmp, states, pstar, n, &feat, &tgt);
    if(rc) return rc;
    float *grad = nullptr, *m1 = c->d_mlp_master + MLP_NPARAM, *m2 = c->d_mlp_master + 2 * MLP_NPARAM;
    float* d_loss = nullptr;
    SPHGPU_CUDA(c, tmp.get(&grad, sizeof(float) * MLP_NPARAM, false));
    SPHGPU_CUDA(c, tmp.get(&d_loss, sizeof(float), false));
    SPHGPU_CUDA(c, cudaMemsetAsync(m1, 0, sizeof(float) * 2 * MLP_NPARAM, c->stream));
    MlpDev md = mlp_device(c);
    const __nv_bfloat16* wt1 = md.w + IMG_W1T;
    const __nv_bfloat16* wt2 = md.w + IMG_W2T;
    auto run_batch = [&](long long base, int bsize, unsigned long long pa, unsigned long long pc) {
        const int tiles = (bsize + 15) / 16;
        const int blocks = std::max(1, std::min(148 * 2, (tiles + 3) / 4));
        k_mlp_train<<<blocks, TBLK, TRAIN_SMEM, c->stream>>>(md, wt1, wt2, feat, tgt, n, base, bsize, pa, pc, grad,
                                                             d_loss);
    };
    SPHGPU_CUDA(c, cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
    if(epochs == 0) {
        SPHGPU_CUDA(c, cudaMemsetAsync(grad, 0, sizeof(float) * MLP_NPARAM, c->stream));
        SPHGPU_CUDA(c, cudaMemsetAsync(d_loss, 0, sizeof(float), c->stream));
        run_batch(0, (int)n, 1ull, 0ull);
        SPHGPU_LAUNCH_CHECK(c, "MLP gradient");
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        if(grad_out) SPHGPU_CUDA(c, cudaMemcpy(grad_out, grad, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost));
        if(loss_history) SPHGPU_CUDA(c, cudaMemcpy(loss_history, d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    }
    uint64_t x = seed | 1;
    int64_t step = 0;
    for(int e = 0; e < epochs; ++e) {
        // a fresh multiplicative permutation of the rows per epoch
        x = x * 6364136223846793005ull + 1442695040888963407ull;
        unsigned long long pa = (x >> 17) % (unsigned long long)n;
        auto gcd = [](unsigned long long a, unsigned long long b) {
            while(b) {
                const unsigned long long r = a % b;
                a = b;
                b = r;
            }
            return a;
        };
        if(pa == 0) pa = 1;
        while(gcd(pa, (unsigned long long)n) != 1) pa = (pa + 1) % (unsigned long long)n;
        const unsigned long long pc = (x >> 33) % (unsigned long long)n;
        double esum = 0.0;
        int nb = 0;
        for(long long base = 0; base < n; base += batch, ++nb) {
            const int bsize = (int)std::min<long long>(batch, n - base);
            SPHGPU_CUDA(c, cudaMemsetAsync(grad, 0, sizeof(float) * MLP_NPARAM, c->stream));
            SPHGPU_CUDA(c, cudaMemsetAsync(d_loss, 0, sizeof(float), c->stream));
            run_batch(base, bsize, pa, pc);
            ++step;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
            k_adam<<<grid_for(MLP_NPARAM, 256), 256, 0, c->stream>>>(c->d_mlp_master, grad, m1, m2, MLP_NPARAM, lr,
                                                                    b1, b2, c1, c2, 1e-8f);
            k_make_image<<<64, 256, 0, c->stream>>>(c->d_mlp_master, static_cast<__nv_bfloat16*>(c->d_mlp),
                                                    reinterpret_cast<float*>(static_cast<char*>(c->d_mlp) +
                                                                             IMG_F32_OFFSET));
            float l = 0.f;
            if(nb % 64 == 0 || base + batch >= n) {
                SPHGPU_CUDA(c, cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
                SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
                esum += l;
            }
        }
        SPHGPU_LAUNCH_CHECK(c, "MLP training");
        if(loss_history) loss_history[e] = (float)(esum / ((nb + 63) / 64));
    }
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    c->mlp_master.resize(MLP_NPARAM);
    SPHGPU_CUDA(c, cudaMemcpy(c->mlp_master.data(), c->d_mlp_master, sizeof(float) * MLP_NPARAM,
                              cudaMemcpyDeviceToHost));
    return SPHGPU_OK;
}

}  // extern "C"
