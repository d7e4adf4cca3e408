// mlp.cuh — the small MLP of the learned MDF warm start.
//
// Network: 64 input features -> 64 -> 64 -> 64 (ReLU) -> 2 outputs, FP32.
// Parameter block (MLP_NP floats, one contiguous device array):
//   [0, 64)        feature means            x' = (x - mean) * inv
//   [64, 128)      feature inverse scales
//   [128, 130)     target scales             the network predicts t * yinv
//   [130, 132)     unused
//   then per layer l = 1..4: W_l [in][out] (row-major, in-major), b_l [out].
// Every layer is evaluated by a whole CTA on a tile of rows held in shared
// memory: thread t owns output column t % 64 and the rows (t / 64) + k * G,
// G = blockDim / 64 groups, so a warp reads one activation row as a broadcast
// and 32 consecutive weights per step.
#pragma once

namespace iblbm {

constexpr int MLP_IN = 64;
constexpr int MLP_H = 64;
constexpr int MLP_OUT = 2;
constexpr int MLP_HDR = 132;
constexpr int MLP_W1 = MLP_HDR;
constexpr int MLP_B1 = MLP_W1 + MLP_IN * MLP_H;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_H * MLP_H;
constexpr int MLP_W4 = MLP_B3 + MLP_H;
constexpr int MLP_B4 = MLP_W4 + MLP_H * MLP_OUT;
constexpr int MLP_NP = MLP_B4 + MLP_OUT;
constexpr int MLP_RPT = 16;  // rows per thread of a layer tile

// One 64-wide layer on `rows` rows (rows <= MLP_RPT * blockDim / 64):
// out[m][o] = act(b[o] + sum_i in[m][i] W[i][o]).  in/out in shared memory,
// row stride 64; W and b in global memory (read through the read-only cache).
__device__ __forceinline__ void mlp_layer64(const float* __restrict__ W, const float* __restrict__ b,
                                            const float* in, float* out, int rows, bool relu)
{
    const int o = threadIdx.x & 63, g = threadIdx.x >> 6, G = blockDim.x >> 6;
    float acc[MLP_RPT];
    const float bo = __ldg(b + o);
#pragma unroll
    for (int k = 0; k < MLP_RPT; ++k) acc[k] = bo;
#pragma unroll 4
    for (int i = 0; i < 64; ++i) {
        const float w = __ldg(W + i * 64 + o);
#pragma unroll
        for (int k = 0; k < MLP_RPT; ++k) {
            const int m = g + k * G;
            if (m < rows) acc[k] += in[m * 64 + i] * w;
        }
    }
#pragma unroll
    for (int k = 0; k < MLP_RPT; ++k) {
        const int m = g + k * G;
        if (m < rows) out[m * 64 + o] = relu ? fmaxf(acc[k], 0.0f) : acc[k];
    }
}

// The 64 -> 2 output layer: threads t < 2 * rows compute row t / 2, output t % 2.
__device__ __forceinline__ void mlp_layer_out(const float* __restrict__ P, const float* in, float* out, int rows)
{
    for (int t = threadIdx.x; t < 2 * rows; t += blockDim.x) {
        const int m = t >> 1, o = t & 1;
        float acc = __ldg(P + MLP_B4 + o);
        for (int i = 0; i < 64; ++i) acc += in[m * 64 + i] * __ldg(P + MLP_W4 + i * 2 + o);
        out[m * 2 + o] = acc;
    }
}

// Forward pass of `rows` normalised rows held in a (row stride 64); b is a
// second buffer of the same size; the 2 outputs per row land in y (shared,
// normalised units).  Ends with the CTA synchronised.
__device__ __forceinline__ void mlp_forward_tile(const float* __restrict__ P, float* a, float* b, float* y, int rows)
{
    mlp_layer64(P + MLP_W1, P + MLP_B1, a, b, rows, true);
    __syncthreads();
    mlp_layer64(P + MLP_W2, P + MLP_B2, b, a, rows, true);
    __syncthreads();
    mlp_layer64(P + MLP_W3, P + MLP_B3, a, b, rows, true);
    __syncthreads();
    mlp_layer_out(P, b, y, rows);
    __syncthreads();
}

}  // namespace iblbm
