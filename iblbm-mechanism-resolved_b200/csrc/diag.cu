// diag.cu — diagnostics reduced on the device: force coefficients into a ring
// buffer and the velocity-convergence error.
//
// The reference reduces its diagnostics on the host at every check
// (iblbm/runtime/loop.py:97-126): Cd / Cl from the IB force summed over the
// whole grid and the mean density (iblbm/diagnostics/core.py:53-113), and the
// relative L2 change of the velocity field (core.py:116-135).  Here each is one
// launch that reads the output step's fields where they are and leaves a few
// doubles in device memory, so a run that needs no stop rule can queue many
// checks (inside CUDA graphs too) and read all their coefficients at once.
//
// Reductions are deterministic: a fixed grid (set by the node count), each
// thread summing a fixed strided set of nodes, a fixed tree in shared memory,
// per-block partials in global memory, and the last block to finish (a ticket
// taken after a fence; it waits on nothing) summing the partials in block order
// and writing the result.  Results differ from numpy's pairwise sums only by
// rounding (about 1e-15 relative on these sums).
#include <cmath>
#include "common.cuh"

namespace iblbm {

constexpr int DIAG_THREADS = 256;
constexpr int DIAG_MAX_BLOCKS = 296;  // two per SM on 148 SMs
constexpr int DIAG_RING_FIELDS = 5;   // Cd, Cl, mean rho, sum Fx, sum Fy

__host__ __device__ inline int diag_blocks(long long n)
{
    const long long b = (n + 8LL * DIAG_THREADS - 1) / (8LL * DIAG_THREADS);
    return (int)(b < 1 ? 1 : (b > DIAG_MAX_BLOCKS ? DIAG_MAX_BLOCKS : b));
}

template <int W>
__device__ __forceinline__ void block_sum(double (&v)[W], double (*red)[DIAG_THREADS])
{
#pragma unroll
    for (int w = 0; w < W; ++w) red[w][threadIdx.x] = v[w];
    __syncthreads();
    for (int s = DIAG_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
#pragma unroll
            for (int w = 0; w < W; ++w) red[w][threadIdx.x] += red[w][threadIdx.x + s];
        }
        __syncthreads();
    }
#pragma unroll
    for (int w = 0; w < W; ++w) v[w] = red[w][0];
}

template <typename T>
__device__ __forceinline__ double ld(const void* p, long long k)
{
    return (double)static_cast<const T*>(p)[k];
}

// Block b sums its strided share of the n densities; the last block adds the
// partials and the force, and writes one ring entry.
template <typename T>
__global__ void __launch_bounds__(DIAG_THREADS) force_coeffs_kernel(const iblbm_force_coeff_args a)
{
    __shared__ double red[2][DIAG_THREADS];
    __shared__ bool last;
    double v[1] = {0.0};
    const long long stride = (long long)gridDim.x * DIAG_THREADS;
    for (long long k = (long long)blockIdx.x * DIAG_THREADS + threadIdx.x; k < a.n_nodes; k += stride)
        v[0] += ld<T>(a.ro, k);
    block_sum<1>(v, red);
    if (threadIdx.x == 0) {
        a.partials[blockIdx.x] = v[0];
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the mean density: partials in block order (a fixed tree over <= 296 values)
    double r[1] = {0.0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += DIAG_THREADS) r[0] += a.partials[b];
    block_sum<1>(r, red);
    // the force: band force of DF / MDF (other grid nodes hold zero), marker force of DFC
    double f[2] = {0.0, 0.0};
    if (a.method == IBLBM_IBM_DFC) {
        for (int l = threadIdx.x; l < a.lb_total; l += DIAG_THREADS) {
            f[0] += a.dfc_force[2 * l];
            f[1] += a.dfc_force[2 * l + 1];
        }
    } else if (a.method != IBLBM_IBM_NONE) {
        const int nb = *a.band_count;
        for (int b = threadIdx.x; b < nb; b += DIAG_THREADS) {
            f[0] += ld<T>(a.band_fib, 2LL * b);
            f[1] += ld<T>(a.band_fib, 2LL * b + 1);
        }
    }
    block_sum<2>(f, red);
    if (threadIdx.x == 0) {
        const double ro_mean = r[0] / (double)a.n_nodes;
        const double denom = ro_mean * (a.u_ref * a.u_ref) * a.lattice_r;
        const int pos = *a.ring_pos;
        double* e = a.ring + (long long)(pos % a.ring_len) * DIAG_RING_FIELDS;
        e[0] = fabs(f[0]) / denom;
        e[1] = f[1] / denom;
        e[2] = ro_mean;
        e[3] = f[0];
        e[4] = f[1];
        *a.ring_pos = pos + 1;
        *a.ticket = 0u;  // ready for the next launch (kernels on one stream run in order)
    }
}

// sum (u - u_prev)^2 and sum u_prev^2 over the n x 2 velocity field; u_prev is
// replaced by u as it is read (the next check's reference field).
template <typename T>
__global__ void __launch_bounds__(DIAG_THREADS) velocity_change_kernel(const iblbm_velocity_change_args a)
{
    __shared__ double red[2][DIAG_THREADS];
    __shared__ bool last;
    double v[2] = {0.0, 0.0};
    const long long m = 2LL * a.n_nodes;
    const long long stride = (long long)gridDim.x * DIAG_THREADS;
    for (long long k = (long long)blockIdx.x * DIAG_THREADS + threadIdx.x; k < m; k += stride) {
        const double u = ld<T>(a.U, k), p = a.U_prev[k];
        const double d = u - p;
        v[0] += d * d;
        v[1] += p * p;
        a.U_prev[k] = u;
    }
    block_sum<2>(v, red);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = v[0];
        a.partials[2 * blockIdx.x + 1] = v[1];
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double r[2] = {0.0, 0.0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += DIAG_THREADS) {
        r[0] += a.partials[2 * b];
        r[1] += a.partials[2 * b + 1];
    }
    block_sum<2>(r, red);
    if (threadIdx.x == 0) {
        a.out[0] = r[0];
        a.out[1] = r[1];
        // iblbm/diagnostics/core.py:116-135: 1.0 when the reference field is zero
        a.out[2] = r[1] == 0.0 ? 1.0 : sqrt(r[0] / r[1]);
        *a.ticket = 0u;
    }
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_diag_partials(int n_nodes) { return 2 * diag_blocks(2LL * n_nodes); }

extern "C" int iblbm_force_coeffs(const iblbm_force_coeff_args* a, void* stream)
{
    if (!a || !a->ro || a->n_nodes < 1 || !a->partials || !a->ticket || !a->ring || a->ring_len < 1 || !a->ring_pos)
        return IBLBM_E_ARG;
    if (a->method == IBLBM_IBM_DFC && (!a->dfc_force || a->lb_total < 0)) return IBLBM_E_ARG;
    if ((a->method == IBLBM_IBM_DF || a->method == IBLBM_IBM_MDF) && (!a->band_fib || !a->band_count))
        return IBLBM_E_ARG;
    const int blocks = diag_blocks(a->n_nodes);
    cudaStream_t s = (cudaStream_t)stream;
    if (a->f32) force_coeffs_kernel<float><<<blocks, DIAG_THREADS, 0, s>>>(*a);
    else force_coeffs_kernel<double><<<blocks, DIAG_THREADS, 0, s>>>(*a);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

extern "C" int iblbm_velocity_change(const iblbm_velocity_change_args* a, void* stream)
{
    if (!a || !a->U || !a->U_prev || a->n_nodes < 1 || !a->partials || !a->ticket || !a->out) return IBLBM_E_ARG;
    const int blocks = diag_blocks(2LL * a->n_nodes);
    cudaStream_t s = (cudaStream_t)stream;
    if (a->f32) velocity_change_kernel<float><<<blocks, DIAG_THREADS, 0, s>>>(*a);
    else velocity_change_kernel<double><<<blocks, DIAG_THREADS, 0, s>>>(*a);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}
