// mlp.cuh — the small MLP of the learned MDF warm start.
//
// Network: 64 input features -> 64 -> 64 -> 64 (ReLU) -> 2 outputs, FP32.
// Parameter block (MLP_NP floats, one contiguous device array):
//   [0, 64)        feature means            x' = (x - mean) * inv
//   [64, 128)      feature inverse scales
//   [128, 130)     target scales             the network predicts t * yinv
//   [130, 132)     unused
//   then per hidden layer l = 1..3: W_l [in][MLP_WLD] (row i holds the 64
//   outputs' weights of input i, then 8 unused floats), b_l [64];
//   then W_4 [64][2], b_4 [2].
// The hidden layers run on the tensor cores: warp-level mma.sync m16n8k8 with
// TF32 operands (rounded to nearest, ties away) and FP32 accumulation.  The
// tiles are 64 or 128 rows, so the warp-level instruction is the fitting one
// (a tcgen05 MMA wants 64-128-row tiles held in tensor memory, whose
// allocation and commit per layer would cost more than these layers take).
// The row stride of 72 floats puts the B-fragment loads (rows k .. k + 3,
// eight consecutive columns) on 32 distinct banks; activation tiles use a
// stride of 68 (MLP_LD) for the A fragments.
#pragma once
#include <cstdint>

namespace iblbm {

constexpr int MLP_IN = 64;
constexpr int MLP_H = 64;
constexpr int MLP_OUT = 2;
constexpr int MLP_HDR = 132;
constexpr int MLP_WLD = 72;  // row stride of the hidden layers' weight matrices
constexpr int MLP_W1 = MLP_HDR;
constexpr int MLP_B1 = MLP_W1 + MLP_IN * MLP_WLD;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_WLD;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_H * MLP_WLD;
constexpr int MLP_W4 = MLP_B3 + MLP_H;
constexpr int MLP_B4 = MLP_W4 + MLP_H * MLP_OUT;
constexpr int MLP_NP = (MLP_B4 + MLP_OUT + 3) / 4 * 4;  // padded to 16 bytes for bulk copies

constexpr int MLP_LD = 68;  // row stride of activation tiles (rows 4 apart fall in different banks)

__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// c (16 x 8, FP32) += a (16 x 8, TF32, row) . b (8 x 8, TF32, col); the PTX
// fragment layout of m16n8k8: lane = 4 g + t holds a (g, t), (g + 8, t),
// (g, t + 4), (g + 8, t + 4); b (t, g), (t + 4, g); c (g, 2t), (g, 2t + 1),
// (g + 8, 2t), (g + 8, 2t + 1).
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc += A (M x 64) . B (64 x 64) for this warp's block: rows 16 (w % (M/16))
// .. + 15 and columns 32 (w / (M/16)) .. + 31 of the M x 64 product (the CTA
// has M / 8 warps).  Operands are read element by element:
// A(m, k) = A[m * as_m + k * as_k], B(k, n) = B[k * bs_k + n * bs_n].
// acc[t] is the 16 x 8 tile of columns 32 (w / (M/16)) + 8 t .. + 7.
template <int M>
__device__ __forceinline__ void tc_gemm64(const float* __restrict__ A, int as_m, int as_k, const float* __restrict__ B,
                                          int bs_k, int bs_n, float (&acc)[4][4])
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    const int m0 = 16 * (warp % (M / 16)), n0 = 32 * (warp / (M / 16));
    const float* a0 = A + (m0 + g) * as_m;
    const float* a1 = A + (m0 + g + 8) * as_m;
    // a compact loop: inside the band kernel this code runs once per step, so
    // unrolled straight-line code would be fetched cold instruction by instruction
#pragma unroll 1
    for (int k0 = 0; k0 < 64; k0 += 8) {
        uint32_t af[4];
        af[0] = to_tf32(a0[(k0 + t4) * as_k]);
        af[1] = to_tf32(a1[(k0 + t4) * as_k]);
        af[2] = to_tf32(a0[(k0 + t4 + 4) * as_k]);
        af[3] = to_tf32(a1[(k0 + t4 + 4) * as_k]);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int n = n0 + 8 * t + g;
            const uint32_t b0 = to_tf32(B[(k0 + t4) * bs_k + n * bs_n]);
            const uint32_t b1 = to_tf32(B[(k0 + t4 + 4) * bs_k + n * bs_n]);
            mma_tf32(acc[t], af, b0, b1);
        }
    }
}

// The output element (row, column) of accumulator entry acc[t][e] of this warp.
template <int M>
__device__ __forceinline__ void tc_coords(int t, int e, int& row, int& col)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    row = 16 * (warp % (M / 16)) + (lane >> 2) + (e >= 2 ? 8 : 0);
    col = 32 * (warp / (M / 16)) + 8 * t + 2 * (lane & 3) + (e & 1);
}

// One 64-wide hidden layer on the M rows of a tile (M / 8 warps, M = 64 or
// 128): out[m][o] = act(b[o] + sum_i in[m][i] W[i][o]) on the tensor cores.
// in/out: tiles of row stride MLP_LD; W (row stride MLP_WLD), b: shared or
// global.  Every row is computed; rows past the valid ones hold whatever the
// input tile holds.
template <int M>
__device__ __forceinline__ void mlp_layer64_tc(const float* W, const float* b, const float* in, float* out, bool relu)
{
    float acc[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int r, c;
            tc_coords<M>(t, e, r, c);
            acc[t][e] = b[c];
        }
    tc_gemm64<M>(in, MLP_LD, 1, W, MLP_WLD, 1, acc);
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int r, c;
            tc_coords<M>(t, e, r, c);
            out[r * MLP_LD + c] = relu ? fmaxf(acc[t][e], 0.0f) : acc[t][e];
        }
}

// The 64 -> 2 output layer (CUDA cores): threads t < 2 * rows compute row t / 2, output t % 2.
__device__ __forceinline__ void mlp_layer_out(const float* P, const float* in, float* out, int rows)
{
    for (int t = threadIdx.x; t < 2 * rows; t += blockDim.x) {
        const int m = t >> 1, o = t & 1;
        float acc = P[MLP_B4 + o];
        for (int i = 0; i < 64; ++i) acc += in[m * MLP_LD + i] * P[MLP_W4 + i * 2 + o];
        out[m * 2 + o] = acc;
    }
}

// Shared-memory room for one hidden layer's weights (stride MLP_WLD).
constexpr int MLP_WBUF = MLP_IN * MLP_WLD;

// Forward pass of a tile of NT / 4 normalised rows held in a (row stride
// MLP_LD); b is a second tile; the 2 outputs of the first `rows` rows land in y
// (normalised units).  NT threads (NT / 32 warps, NT / 4 rows).  With wbuf
// (MLP_WBUF floats of shared memory, 16-byte aligned) each hidden layer's
// weights are first copied there from P, so the tensor-core loop reads its B
// operands from shared memory instead of waiting on L2.  Ends with the CTA
// synchronised.
template <int NT>
__device__ __forceinline__ void mlp_forward_tile(const float* P, float* a, float* b, float* y, int rows,
                                                 float* wbuf = nullptr)
{
    constexpr int M = NT / 4;
    float* in = a;
    float* out = b;
#pragma unroll 1
    for (int l = 0; l < 3; ++l) {
        const float* w = P + MLP_W1 + l * (MLP_W2 - MLP_W1);
        const float* bl = P + MLP_B1 + l * (MLP_B2 - MLP_B1);
        if (wbuf) {
            const float4* src = reinterpret_cast<const float4*>(w);
            float4* dst = reinterpret_cast<float4*>(wbuf);
            for (int e = threadIdx.x; e < MLP_WBUF / 4; e += NT) dst[e] = src[e];
            __syncthreads();
            w = wbuf;
        }
        mlp_layer64_tc<M>(w, bl, in, out, true);
        __syncthreads();
        float* t = in;
        in = out;
        out = t;
    }
    mlp_layer_out(P, in, y, rows);
    __syncthreads();
}

}  // namespace iblbm
