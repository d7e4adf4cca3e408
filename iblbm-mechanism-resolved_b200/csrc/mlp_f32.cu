// mlp_f32.cu — fused training and inference kernels of the learned MDF warm start.
//
// Training step (one launch): every CTA takes 64 samples, runs the forward pass
// keeping all activations in shared memory, back-propagates the mean squared
// error, and adds its weight and bias gradients into one global gradient
// buffer; the last CTA to finish (counted with an atomic ticket after a memory
// fence, no waiting) applies the Adam update to every parameter and clears the
// buffer for the next step.  Inference: 128 samples per CTA.
#include <cstdint>
#include "mlp.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int TRAIN_ROWS = 64;
constexpr int TRAIN_THREADS = 256;
constexpr int INFER_THREADS = 512;
constexpr int INFER_ROWS = INFER_THREADS / 4;  // 128
constexpr float ADAM_B1 = 0.9f, ADAM_B2 = 0.999f, ADAM_EPS = 1e-8f;

// Smem layout of the training kernel (floats): A0..A3 activations, two delta
// buffers, the staged weight matrix (row stride 65), outputs and output deltas.
static_assert(TRAIN_ROWS == TRAIN_THREADS / 4, "one layer tile per CTA");
constexpr int TR_A = TRAIN_ROWS * MLP_LD;
constexpr size_t TRAIN_SMEM = sizeof(float) * (size_t)(4 * TR_A + 2 * TR_A + 64 * 65 + 2 * TRAIN_ROWS * 2);

// Normalised input tile: rows beyond n are zero.
__device__ __forceinline__ void load_inputs(const float* __restrict__ P, const float* __restrict__ X, int r0, int rows,
                                            int nrows_tile, float* a)
{
    for (int e = threadIdx.x; e < nrows_tile * 64; e += blockDim.x) {
        const int m = e >> 6, i = e & 63;
        a[m * MLP_LD + i] = m < rows ? (X[(size_t)(r0 + m) * 64 + i] - __ldg(P + i)) * __ldg(P + 64 + i) : 0.0f;
    }
}

// gW[i][o] += sum_m A[m][i] D[m][o], gb[o] += sum_m D[m][o]  (64 x 64, TRAIN_ROWS rows)
__device__ __forceinline__ void grad_w64(const float* A, const float* D, float* gW, float* gb)
{
    const int o = threadIdx.x & 63, g = threadIdx.x >> 6, G = blockDim.x >> 6;
    float acc[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[k] = 0.0f;
    for (int m = 0; m < TRAIN_ROWS; ++m) {
        const float d = D[m * MLP_LD + o];
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[k] += A[m * MLP_LD + g + k * G] * d;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) atomicAdd(gW + (g + k * G) * 64 + o, acc[k]);
    if (threadIdx.x < 64) {
        float s = 0.0f;
        for (int m = 0; m < TRAIN_ROWS; ++m) s += D[m * MLP_LD + threadIdx.x];
        atomicAdd(gb + threadIdx.x, s);
    }
}

// Din[m][i] = (A[m][i] > 0) * sum_o W[i][o] Dout[m][o] with W staged in sW (stride 65)
__device__ __forceinline__ void backprop64(const float* __restrict__ W, float* sW, const float* Dout, const float* A,
                                           float* Din)
{
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) sW[(e >> 6) * 65 + (e & 63)] = __ldg(W + e);
    __syncthreads();
    const int i = threadIdx.x & 63, g = threadIdx.x >> 6, G = blockDim.x >> 6;
    float acc[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[k] = 0.0f;
    for (int o = 0; o < 64; ++o) {
        const float w = sW[i * 65 + o];
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[k] += Dout[(g + k * G) * MLP_LD + o] * w;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int m = g + k * G;
        Din[m * MLP_LD + i] = A[m * MLP_LD + i] > 0.0f ? acc[k] : 0.0f;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(TRAIN_THREADS) mlp_train_kernel(float* __restrict__ P, float* __restrict__ am,
                                                                  float* __restrict__ av, float* __restrict__ grad,
                                                                  unsigned* __restrict__ ticket,
                                                                  const float* __restrict__ X,
                                                                  const float* __restrict__ T, int n, float lr,
                                                                  float c1, float c2, float* __restrict__ loss,
                                                                  int apply)
{
    extern __shared__ __align__(16) float sm[];
    float* A0 = sm;
    float* A1 = A0 + TR_A;
    float* A2 = A1 + TR_A;
    float* A3 = A2 + TR_A;
    float* Da = A3 + TR_A;
    float* Db = Da + TR_A;
    float* sW = Db + TR_A;
    float* Y = sW + 64 * 65;
    float* D4 = Y + TRAIN_ROWS * 2;
    __shared__ int s_last;
    const int r0 = blockIdx.x * TRAIN_ROWS, rows = min(TRAIN_ROWS, n - r0);
    load_inputs(P, X, r0, rows, TRAIN_ROWS, A0);
    __syncthreads();
    mlp_layer64<TRAIN_THREADS>(P + MLP_W1, P + MLP_B1, A0, A1, true);
    __syncthreads();
    mlp_layer64<TRAIN_THREADS>(P + MLP_W2, P + MLP_B2, A1, A2, true);
    __syncthreads();
    mlp_layer64<TRAIN_THREADS>(P + MLP_W3, P + MLP_B3, A2, A3, true);
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
    if (loss) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) part += __shfl_xor_sync(0xffffffffu, part, s);
        if ((threadIdx.x & 31) == 0 && part != 0.0f) atomicAdd(loss, part / (float)n);
    }
    __syncthreads();
    // output layer: gW4[i][o] = sum_m A3[m][i] D4[m][o], gb4; D3 = (D4 W4^T) * (A3 > 0)
    for (int e = threadIdx.x; e < 64 * 2; e += blockDim.x) {
        const int i = e >> 1, o = e & 1;
        float s = 0.0f;
        for (int m = 0; m < TRAIN_ROWS; ++m) s += A3[m * MLP_LD + i] * D4[m * 2 + o];
        atomicAdd(grad + MLP_W4 + e, s);
    }
    if (threadIdx.x < 2) {
        float s = 0.0f;
        for (int m = 0; m < TRAIN_ROWS; ++m) s += D4[m * 2 + threadIdx.x];
        atomicAdd(grad + MLP_B4 + threadIdx.x, s);
    }
    for (int e = threadIdx.x; e < TRAIN_ROWS * 64; e += blockDim.x) {
        const int m = e >> 6, i = e & 63;
        const float s = __ldg(P + MLP_W4 + i * 2) * D4[m * 2] + __ldg(P + MLP_W4 + i * 2 + 1) * D4[m * 2 + 1];
        Da[m * MLP_LD + i] = A3[m * MLP_LD + i] > 0.0f ? s : 0.0f;
    }
    __syncthreads();
    grad_w64(A2, Da, grad + MLP_W3, grad + MLP_B3);
    backprop64(P + MLP_W3, sW, Da, A2, Db);
    grad_w64(A1, Db, grad + MLP_W2, grad + MLP_B2);
    backprop64(P + MLP_W2, sW, Db, A1, Da);
    grad_w64(A0, Da, grad + MLP_W1, grad + MLP_B1);
    if (!apply) return;
    // the last CTA applies Adam to the summed gradients and clears them
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int p = MLP_HDR + threadIdx.x; p < MLP_NP; p += blockDim.x) {
        const float gp = __ldcg(grad + p);
        const float m = ADAM_B1 * am[p] + (1.0f - ADAM_B1) * gp;
        const float v = ADAM_B2 * av[p] + (1.0f - ADAM_B2) * gp * gp;
        am[p] = m;
        av[p] = v;
        P[p] -= lr * (m * c1) / (sqrtf(v * c2) + ADAM_EPS);
        grad[p] = 0.0f;
    }
    if (threadIdx.x == 0) *ticket = 0u;
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

extern "C" int iblbm_mlp_infer(const float* params, const float* x, int n, float* y, void* stream)
{
    if (!params || !x || !y || n < 0) return IBLBM_E_ARG;
    if (n == 0) return IBLBM_OK;
    const size_t smem = sizeof(float) * (size_t)(2 * INFER_ROWS * MLP_LD + INFER_ROWS * 2);
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return IBLBM_E_LAUNCH;
        configured = true;
    }
    mlp_infer_kernel<<<(n + INFER_ROWS - 1) / INFER_ROWS, INFER_THREADS, smem, (cudaStream_t)stream>>>(params, x, n,
                                                                                                      y);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

extern "C" int iblbm_mlp_train_step(float* params, float* adam_m, float* adam_v, float* grad, unsigned* ticket,
                                    const float* x, const float* t, int n, float lr, int step, float* loss,
                                    int apply, void* stream)
{
    if (!params || !grad || !ticket || !x || !t || n < 1 || step < 1) return IBLBM_E_ARG;
    if (apply && (!adam_m || !adam_v)) return IBLBM_E_ARG;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM) !=
            cudaSuccess)
            return IBLBM_E_LAUNCH;
        configured = true;
    }
    // Adam bias corrections 1 / (1 - beta^step)
    const float c1 = (float)(1.0 / (1.0 - pow((double)ADAM_B1, step)));
    const float c2 = (float)(1.0 / (1.0 - pow((double)ADAM_B2, step)));
    mlp_train_kernel<<<(n + TRAIN_ROWS - 1) / TRAIN_ROWS, TRAIN_THREADS, TRAIN_SMEM, (cudaStream_t)stream>>>(
        params, adam_m, adam_v, grad, ticket, x, t, n, lr, c1, c2, loss, apply);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}
