// mlp_f32.cu — fused training and inference kernels of the learned MDF warm start.
//
// Training step (two launches, no atomics, the same bits on every run): every
// CTA of the first kernel takes 64 samples, runs the forward pass keeping all
// activations in shared memory, back-propagates the mean squared error and
// writes its own weight and bias gradients (and its share of the loss) to its
// slot of the gradient buffer; the second kernel sums the CTAs' slots in CTA
// order for every parameter and applies the Adam update (or leaves the summed
// gradient).  The three 64 x 64 layers' forward products, their weight
// gradients (A^T D) and the back-propagated deltas (D W^T) all run on the
// tensor cores (mlp.cuh tc_gemm64); the 64 -> 2 output layer stays on CUDA
// cores.  Inference: 128 samples per CTA.
#include <cstdint>
#include "common.cuh"
#include "mlp.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int TRAIN_ROWS = 64;
constexpr int TRAIN_THREADS = 256;  // 8 warps: the 64 x 64 products in 16 x 32 blocks
constexpr int INFER_THREADS = 512;
constexpr int INFER_ROWS = INFER_THREADS / 4;  // 128
constexpr int REDUCE_THREADS = 256;
constexpr int GRAD_SLOT = MLP_NP + 4;  // one CTA's gradient, then its loss, padded to 16 bytes
constexpr float ADAM_B1 = 0.9f, ADAM_B2 = 0.999f, ADAM_EPS = 1e-8f;

static_assert(TRAIN_ROWS == TRAIN_THREADS / 4, "one layer tile per CTA");
constexpr int TR_A = TRAIN_ROWS * MLP_LD;
constexpr size_t TRAIN_SMEM = sizeof(float) * (size_t)(4 * TR_A + 2 * TR_A + 2 * TRAIN_ROWS * 2 + 32);

// Normalised input tile: rows beyond n are zero.
__device__ __forceinline__ void load_inputs(const float* __restrict__ P, const float* __restrict__ X, int r0, int rows,
                                            int nrows_tile, float* a)
{
    for (int e = threadIdx.x; e < nrows_tile * 64; e += blockDim.x) {
        const int m = e >> 6, i = e & 63;
        a[m * MLP_LD + i] = m < rows ? (X[(size_t)(r0 + m) * 64 + i] - __ldg(P + i)) * __ldg(P + 64 + i) : 0.0f;
    }
}

// g[W + i * MLP_WLD + o] = sum_m A[m][i] D[m][o] (tensor cores), g[b + o] =
// sum_m D[m][o], and the 8 unused floats of every weight row are zero.
__device__ __forceinline__ void grad_layer(const float* A, const float* D, float* g, int W, int b)
{
    float acc[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[t][e] = 0.0f;
    // C(i, o) = sum_m A(i, m) B(m, o) with A(i, m) = A[m][i], B(m, o) = D[m][o]
    tc_gemm64<64>(A, 1, MLP_LD, D, MLP_LD, 1, acc);
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int i, o;
            tc_coords<64>(t, e, i, o);
            g[W + i * MLP_WLD + o] = acc[t][e];
        }
    for (int e = threadIdx.x; e < 64 * (MLP_WLD - 64); e += blockDim.x)
        g[W + (e >> 3) * MLP_WLD + 64 + (e & 7)] = 0.0f;
    if (threadIdx.x < 64) {
        float s = 0.0f;
        for (int m = 0; m < TRAIN_ROWS; ++m) s += D[m * MLP_LD + threadIdx.x];
        g[b + threadIdx.x] = s;
    }
}

// Din[m][i] = (A[m][i] > 0) * sum_o Dout[m][o] W[i][o] (tensor cores)
__device__ __forceinline__ void backprop_layer(const float* __restrict__ W, const float* Dout, const float* A, float* Din)
{
    float acc[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[t][e] = 0.0f;
    // C(m, i) = sum_o A(m, o) B(o, i) with A(m, o) = Dout[m][o], B(o, i) = W[i][o]
    tc_gemm64<64>(Dout, MLP_LD, 1, W, 1, MLP_WLD, acc);
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int m, i;
            tc_coords<64>(t, e, m, i);
            Din[m * MLP_LD + i] = A[m * MLP_LD + i] > 0.0f ? acc[t][e] : 0.0f;
        }
}

__global__ void __launch_bounds__(TRAIN_THREADS) mlp_grad_kernel(const float* __restrict__ P, float* __restrict__ grad,
                                                                 const float* __restrict__ X,
                                                                 const float* __restrict__ T, int n)
{
    extern __shared__ __align__(16) float sm[];
    float* A0 = sm;
    float* A1 = A0 + TR_A;
    float* A2 = A1 + TR_A;
    float* A3 = A2 + TR_A;
    float* Da = A3 + TR_A;
    float* Db = Da + TR_A;
    float* Y = Db + TR_A;
    float* D4 = Y + TRAIN_ROWS * 2;
    float* red = D4 + TRAIN_ROWS * 2;  // 8 warp partial losses
    float* g = grad + (size_t)GRAD_SLOT * (1 + blockIdx.x);
    const int r0 = blockIdx.x * TRAIN_ROWS, rows = min(TRAIN_ROWS, n - r0);
    load_inputs(P, X, r0, rows, TRAIN_ROWS, A0);
    __syncthreads();
    mlp_layer64_tc<TRAIN_ROWS>(P + MLP_W1, P + MLP_B1, A0, A1, true);
    __syncthreads();
    mlp_layer64_tc<TRAIN_ROWS>(P + MLP_W2, P + MLP_B2, A1, A2, true);
    __syncthreads();
    mlp_layer64_tc<TRAIN_ROWS>(P + MLP_W3, P + MLP_B3, A2, A3, true);
    __syncthreads();
    mlp_layer_out(P, A3, Y, TRAIN_ROWS);
    __syncthreads();
    // loss = (1/n) sum (y - t * yinv)^2, dL/dy = 2 (y - t * yinv) / n
    float part = 0.0f;
    for (int e = threadIdx.x; e < TRAIN_ROWS * 2; e += blockDim.x) {
        const int m = e >> 1, o = e & 1;
        float d = 0.0f;
        if (m < rows) {
            const float r = Y[e] - T[(size_t)(r0 + m) * 2 + o] * __ldg(P + 128 + o);
            part += r * r;
            d = 2.0f * r / (float)n;
        }
        D4[e] = d;
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) part += __shfl_xor_sync(0xffffffffu, part, s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        float L = 0.0f;
        for (int w = 0; w < TRAIN_THREADS / 32; ++w) L += red[w];  // warps in order
        g[MLP_NP] = L / (float)n;
    }
    // output layer: gW4[i][o] = sum_m A3[m][i] D4[m][o], gb4; D3 = (D4 W4^T) * (A3 > 0)
    for (int e = threadIdx.x; e < 64 * 2; e += blockDim.x) {
        const int i = e >> 1, o = e & 1;
        float s = 0.0f;
        for (int m = 0; m < TRAIN_ROWS; ++m) s += A3[m * MLP_LD + i] * D4[m * 2 + o];
        g[MLP_W4 + e] = s;
    }
    if (threadIdx.x < 2) {
        float s = 0.0f;
        for (int m = 0; m < TRAIN_ROWS; ++m) s += D4[m * 2 + threadIdx.x];
        g[MLP_B4 + threadIdx.x] = s;
    }
    for (int p = MLP_B4 + 2 + threadIdx.x; p < MLP_NP; p += blockDim.x) g[p] = 0.0f;
    for (int e = threadIdx.x; e < TRAIN_ROWS * 64; e += blockDim.x) {
        const int m = e >> 6, i = e & 63;
        const float s = __ldg(P + MLP_W4 + i * 2) * D4[m * 2] + __ldg(P + MLP_W4 + i * 2 + 1) * D4[m * 2 + 1];
        Da[m * MLP_LD + i] = A3[m * MLP_LD + i] > 0.0f ? s : 0.0f;
    }
    __syncthreads();
    grad_layer(A2, Da, g, MLP_W3, MLP_B3);
    backprop_layer(P + MLP_W3, Da, A2, Db);
    __syncthreads();
    grad_layer(A1, Db, g, MLP_W2, MLP_B2);
    backprop_layer(P + MLP_W2, Db, A1, Da);
    __syncthreads();
    grad_layer(A0, Da, g, MLP_W1, MLP_B1);
}

// Sum of the CTAs' gradient slots in CTA order; then Adam (apply) or the sum
// into grad[0 .. MLP_NP) (header entries zero).  Block 0 adds the loss.
__global__ void __launch_bounds__(REDUCE_THREADS) mlp_reduce_kernel(float* __restrict__ P, float* __restrict__ am,
                                                                    float* __restrict__ av, float* __restrict__ grad,
                                                                    int nslots, float lr, float c1, float c2,
                                                                    float* __restrict__ loss, int apply)
{
    const int p = blockIdx.x * REDUCE_THREADS + threadIdx.x;
    if (p < MLP_NP) {
        float gp = 0.0f;
        if (p >= MLP_HDR)
            for (int c = 0; c < nslots; ++c) gp += grad[(size_t)GRAD_SLOT * (1 + c) + p];
        if (apply) {
            if (p >= MLP_HDR) {
                const float m = ADAM_B1 * am[p] + (1.0f - ADAM_B1) * gp;
                const float v = ADAM_B2 * av[p] + (1.0f - ADAM_B2) * gp * gp;
                am[p] = m;
                av[p] = v;
                P[p] -= lr * (m * c1) / (sqrtf(v * c2) + ADAM_EPS);
            }
        } else {
            grad[p] = gp;
        }
    }
    if (loss && blockIdx.x == 0 && threadIdx.x == 0) {
        float L = 0.0f;
        for (int c = 0; c < nslots; ++c) L += grad[(size_t)GRAD_SLOT * (1 + c) + MLP_NP];
        *loss += L;
    }
}

__global__ void __launch_bounds__(INFER_THREADS) mlp_infer_kernel(const float* __restrict__ P,
                                                                  const float* __restrict__ X, int n,
                                                                  float* __restrict__ Yout)
{
    extern __shared__ __align__(16) float sm[];
    float* a = sm;
    float* b = a + INFER_ROWS * MLP_LD;
    float* y = b + INFER_ROWS * MLP_LD;
    const int r0 = blockIdx.x * INFER_ROWS, rows = min(INFER_ROWS, n - r0);
    load_inputs(P, X, r0, rows, INFER_ROWS, a);
    __syncthreads();
    mlp_forward_tile<INFER_THREADS>(P, a, b, y, rows);
    for (int e = threadIdx.x; e < rows * 2; e += blockDim.x) Yout[(size_t)r0 * 2 + e] = y[e] / __ldg(P + 128 + (e & 1));
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_mlp_param_count(void) { return MLP_NP; }

extern "C" int iblbm_mlp_grad_floats(int n)
{
    if (n < 1) return GRAD_SLOT;
    return GRAD_SLOT * (1 + (n + TRAIN_ROWS - 1) / TRAIN_ROWS);
}

extern "C" int iblbm_mlp_infer(const float* params, const float* x, int n, float* y, void* stream)
{
    if (!params || !x || !y || n < 0) return IBLBM_E_ARG;
    if (n == 0) return IBLBM_OK;
    const size_t smem = sizeof(float) * (size_t)(2 * INFER_ROWS * MLP_LD + INFER_ROWS * 2);
    if (iblbm::smem_limit_once<mlp_infer_kernel>((int)smem) != cudaSuccess) return IBLBM_E_LAUNCH;
    mlp_infer_kernel<<<(n + INFER_ROWS - 1) / INFER_ROWS, INFER_THREADS, smem, (cudaStream_t)stream>>>(params, x, n,
                                                                                                      y);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

extern "C" int iblbm_mlp_train_step(float* params, float* adam_m, float* adam_v, float* grad, const float* x,
                                    const float* t, int n, float lr, int step, float* loss, int apply, void* stream)
{
    if (!params || !grad || !x || !t || n < 1 || step < 1) return IBLBM_E_ARG;
    if (apply && (!adam_m || !adam_v)) return IBLBM_E_ARG;
    if (iblbm::smem_limit_once<mlp_grad_kernel>((int)TRAIN_SMEM) != cudaSuccess) return IBLBM_E_LAUNCH;
    // Adam bias corrections 1 / (1 - beta^step)
    const float c1 = (float)(1.0 / (1.0 - pow((double)ADAM_B1, step)));
    const float c2 = (float)(1.0 / (1.0 - pow((double)ADAM_B2, step)));
    const int nslots = (n + TRAIN_ROWS - 1) / TRAIN_ROWS;
    cudaStream_t s = (cudaStream_t)stream;
    mlp_grad_kernel<<<nslots, TRAIN_THREADS, TRAIN_SMEM, s>>>(params, grad, x, t, n);
    mlp_reduce_kernel<<<(MLP_NP + REDUCE_THREADS - 1) / REDUCE_THREADS, REDUCE_THREADS, 0, s>>>(
        params, adam_m, adam_v, grad, nslots, lr, c1, c2, loss, apply);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}
