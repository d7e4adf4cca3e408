// mlp.cuh — the small MLP of the learned MDF warm start.
//
// Network: 64 input features -> 64 -> 64 -> 64 (ReLU) -> 2 outputs, FP32.
// Parameter block (MLP_NP floats, one contiguous device array):
//   [0, 64)        feature means            x' = (x - mean) * inv
//   [64, 128)      feature inverse scales
//   [128, 130)     target scales             the network predicts t * yinv
//   [130, 132)     unused
//   then per layer l = 1..4: W_l [in][out] (row-major, in-major), b_l [out].
// Every layer is evaluated by a whole CTA of NT threads on a tile of NT / 4
// rows held in shared memory, each thread a 4 x 4 block of outputs.
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
constexpr int MLP_NP = (MLP_B4 + MLP_OUT + 3) / 4 * 4;  // padded to 16 bytes for bulk copies

constexpr int MLP_LD = 68;  // row stride of activation tiles (rows 4 apart fall in different banks)

// One 64-wide layer on the NT / 4 rows of a tile: out[m][o] = act(b[o] +
// sum_i in[m][i] W[i][o]).  Thread t computes a 4 x 4 block: columns
// 4 (t % 16) .. +3 (one 16-byte weight load per i) and rows 4 (t / 16) .. +3.
// in/out: shared-memory tiles of row stride MLP_LD; W, b: shared or global.
// Every row is computed; rows past the valid ones hold whatever the tile holds.
template <int NT>
__device__ __forceinline__ void mlp_layer64(const float* W, const float* b, const float* in, float* out, bool relu)
{
    const int cg = threadIdx.x & 15, rg = threadIdx.x >> 4;
    const float4 bb = *reinterpret_cast<const float4*>(b + 4 * cg);
    float acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        acc[r][0] = bb.x; acc[r][1] = bb.y; acc[r][2] = bb.z; acc[r][3] = bb.w;
    }
    const float* in0 = in + 4 * rg * MLP_LD;
#pragma unroll 4
    for (int i = 0; i < 64; ++i) {
        const float4 w = *reinterpret_cast<const float4*>(W + i * 64 + 4 * cg);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float x = in0[r * MLP_LD + i];
            acc[r][0] += x * w.x; acc[r][1] += x * w.y; acc[r][2] += x * w.z; acc[r][3] += x * w.w;
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float v = acc[r][c];
            out[(4 * rg + r) * MLP_LD + 4 * cg + c] = relu ? fmaxf(v, 0.0f) : v;
        }
}

// The 64 -> 2 output layer: threads t < 2 * rows compute row t / 2, output t % 2.
__device__ __forceinline__ void mlp_layer_out(const float* P, const float* in, float* out, int rows)
{
    for (int t = threadIdx.x; t < 2 * rows; t += blockDim.x) {
        const int m = t >> 1, o = t & 1;
        float acc = P[MLP_B4 + o];
        for (int i = 0; i < 64; ++i) acc += in[m * MLP_LD + i] * P[MLP_W4 + i * 2 + o];
        out[m * 2 + o] = acc;
    }
}

// Forward pass of a tile of NT / 4 normalised rows held in a (row stride
// MLP_LD); b is a second tile; the 2 outputs of the first `rows` rows land in y
// (normalised units).  Ends with the CTA synchronised.
template <int NT>
__device__ __forceinline__ void mlp_forward_tile(const float* P, float* a, float* b, float* y, int rows)
{
    mlp_layer64<NT>(P + MLP_W1, P + MLP_B1, a, b, true);
    __syncthreads();
    mlp_layer64<NT>(P + MLP_W2, P + MLP_B2, b, a, true);
    __syncthreads();
    mlp_layer64<NT>(P + MLP_W3, P + MLP_B3, a, b, true);
    __syncthreads();
    mlp_layer_out(P, b, y, rows);
    __syncthreads();
}

}  // namespace iblbm
