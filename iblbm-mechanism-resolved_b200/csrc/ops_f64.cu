// ops_f64.cu — one-op-per-call kernels on the reference's AoS layout
// (f[n*9 + q]), the drop-in for iblbm/gpu_kernels.py's Python wrappers, plus the
// AoS <-> pitched-SoA converters of the fused engine.  FP64, -fmad=false, same
// expression order as the reference CPU path.
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int OPS_BLOCK = 256;

__global__ void feq_kernel(const double* __restrict__ ro, const double* __restrict__ U, int N, int incomp,
                           double* __restrict__ feq)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double out[9];
    feq_all(ro[n], U[2 * n], U[2 * n + 1], incomp != 0, out);
#pragma unroll
    for (int q = 0; q < 9; ++q) feq[9 * (long long)n + q] = out[q];
}

__global__ void macro_kernel(const double* __restrict__ f, int N, int incomp, double* __restrict__ ro,
                             double* __restrict__ U)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double v[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) v[q] = f[9 * (long long)n + q];
    double r, a, b;
    macro_seq(v, incomp != 0, r, a, b);
    ro[n] = r;
    U[2 * n] = a;
    U[2 * n + 1] = b;
}

// bgk.py:25-40
__global__ void bgk_kernel(const double* __restrict__ fs, const double* __restrict__ feq,
                           const double* __restrict__ U, const double* __restrict__ fib, int N, double inv_tau,
                           double guo_pref, double dt, double* __restrict__ f)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double u0 = U[2 * n], u1 = U[2 * n + 1], F0 = fib[2 * n], F1 = fib[2 * n + 1];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double ex = (double)ex_(q), ey = (double)ey_(q);
        const double ax = ex - u0, ay = ey - u1;
        const double eU = ex * u0 + ey * u1;
        const double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
        const double F_ni = guo_pref * w_(q) * term;
        const long long k = 9 * (long long)n + q;
        f[k] = fs[k] - inv_tau * (fs[k] - feq[k]) + F_ni * dt;
    }
}

// trt.py:38-67
__global__ void trt_kernel(const double* __restrict__ fs, const double* __restrict__ feq,
                           const double* __restrict__ U, const double* __restrict__ fib, int N, double sp,
                           double sm, double dt, double* __restrict__ f)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double u0 = U[2 * n], u1 = U[2 * n + 1], F0 = fib[2 * n], F1 = fib[2 * n + 1];
    double v[9], e[9], bare[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        v[q] = fs[9 * (long long)n + q];
        e[q] = feq[9 * (long long)n + q];
        const double ex = (double)ex_(q), ey = (double)ey_(q);
        const double ax = ex - u0, ay = ey - u1;
        const double eU = ex * u0 + ey * u1;
        const double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
        bare[q] = w_(q) * term;
    }
    const double gp = 1.0 - 0.5 * sp, gm = 1.0 - 0.5 * sm;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int o = opp_(q);
        const double fp = 0.5 * (v[q] + v[o]), fm = 0.5 * (v[q] - v[o]);
        const double ep = 0.5 * (e[q] + e[o]), em = 0.5 * (e[q] - e[o]);
        const double coll = (sp * (fp - ep) + sm * (fm - em));
        const double bp = 0.5 * (bare[q] + bare[o]), bm = 0.5 * (bare[q] - bare[o]);
        const double F_ni = gp * bp + gm * bm;
        f[9 * (long long)n + q] = v[q] - coll + F_ni * dt;
    }
}

struct S9 { double s[9]; };

// cm_mrt.py:52-165 (always with the forcing moments, as the reference)
__global__ void cmmrt_kernel(const double* __restrict__ fs, const double* __restrict__ U,
                             const double* __restrict__ fib, int N, S9 S, double dt, double* __restrict__ fo)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double ux = U[2 * n], uy = U[2 * n + 1], F0 = fib[2 * n], F1 = fib[2 * n + 1];
    double cm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Fc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double val = fs[9 * (long long)n + q];
        const double ex = (double)ex_(q), ey = (double)ey_(q);
        const double cix = ex - ux, ciy = ey - uy, cix2 = cix * cix, ciy2 = ciy * ciy;
        cm[0] += val; cm[1] += val * cix; cm[2] += val * ciy; cm[3] += val * cix2; cm[4] += val * ciy2;
        cm[5] += val * cix * ciy; cm[6] += val * cix2 * ciy; cm[7] += val * cix * ciy2; cm[8] += val * cix2 * ciy2;
        const double eU = ex * ux + ey * uy;
        const double term = ((3.0 * cix + 9.0 * eU * ex) * F0 + (3.0 * ciy + 9.0 * eU * ey) * F1);
        const double Fb = w_(q) * term;
        Fc[0] += Fb; Fc[1] += Fb * cix; Fc[2] += Fb * ciy; Fc[3] += Fb * cix2; Fc[4] += Fb * ciy2;
        Fc[5] += Fb * cix * ciy; Fc[6] += Fb * cix2 * ciy; Fc[7] += Fb * cix * ciy2; Fc[8] += Fb * cix2 * ciy2;
    }
    const double rho = cm[0], cs2 = 1.0 / 3.0, cs4 = 1.0 / 9.0;
    const double eq[9] = {rho, 0.0, 0.0, rho * cs2, rho * cs2, 0.0, 0.0, 0.0, rho * cs4};
    double c[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) c[m] = cm[m] - S.s[m] * (cm[m] - eq[m]) + (1.0 - 0.5 * S.s[m]) * Fc[m] * dt;
    const double ux2 = ux * ux, uy2 = uy * uy;
    const double k0 = c[0];
    const double k1 = c[1] + ux * c[0];
    const double k2 = c[2] + uy * c[0];
    const double k3 = c[3] + 2.0 * ux * c[1] + ux2 * c[0];
    const double k4 = c[4] + 2.0 * uy * c[2] + uy2 * c[0];
    const double k5 = c[5] + uy * c[1] + ux * c[2] + ux * uy * c[0];
    const double k6 = (c[6] + uy * c[3] + 2.0 * ux * c[5] + 2.0 * ux * uy * c[1] + ux2 * c[2] + ux2 * uy * c[0]);
    const double k7 = (c[7] + 2.0 * uy * c[5] + ux * c[4] + 2.0 * ux * uy * c[2] + uy2 * c[1] + ux * uy2 * c[0]);
    const double k8 = (c[8] + 2.0 * uy * c[6] + uy2 * c[3] + 2.0 * ux * c[7] + 4.0 * ux * uy * c[5] +
                       2.0 * ux * uy2 * c[1] + ux2 * c[4] + 2.0 * ux2 * uy * c[2] + ux2 * uy2 * c[0]);
    double* o = fo + 9 * (long long)n;
    o[0] = k0 - k3 - k4 + k8;
    o[1] = 0.5 * (k1 + k3 - k7 - k8);
    o[2] = 0.5 * (k2 + k4 - k6 - k8);
    o[3] = 0.5 * (-k1 + k3 + k7 - k8);
    o[4] = 0.5 * (-k2 + k4 + k6 - k8);
    o[5] = 0.25 * (k5 + k6 + k7 + k8);
    o[6] = 0.25 * (-k5 + k6 - k7 + k8);
    o[7] = 0.25 * (k5 - k6 - k7 + k8);
    o[8] = 0.25 * (-k5 - k6 + k7 + k8);
}

// streaming.py:38-77 (out-of-lattice sources keep the previous value)
__global__ void stream_kernel(const double* __restrict__ fold, const double* __restrict__ f, int nx, int ny,
                              double* __restrict__ fnew)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= nx) return;
    const long long n = (long long)j * nx + i;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int si = i - ex_(q), sj = j - ey_(q);
        const bool in = si >= 0 && si < nx && sj >= 0 && sj < ny;
        fnew[9 * n + q] = in ? f[9 * ((long long)sj * nx + si) + q] : fold[9 * n + q];
    }
}

// dispatch.py:18-33 (CPU branch arithmetic)
__global__ void vcorr_kernel(double* __restrict__ U, const double* __restrict__ fib, const double* __restrict__ ro,
                             int N, double dt, int incomp)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    for (int c = 0; c < 2; ++c) {
        if (incomp) U[2 * n + c] = U[2 * n + c] + 0.5 * fib[2 * n + c] * dt;
        else U[2 * n + c] = U[2 * n + c] + fib[2 * n + c] * dt / (2.0 * ro[n]);
    }
}

__global__ void aos_to_soa_kernel(const double* __restrict__ aos, Geom g, double* __restrict__ soa)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= g.nx) return;
    const long long n = (long long)j * g.nx + i;
#pragma unroll
    for (int q = 0; q < 9; ++q) soa[q * g.qstride + (long long)j * g.pitch + i] = aos[9 * n + q];
}

__global__ void soa_to_aos_kernel(const double* __restrict__ soa, Geom g, double* __restrict__ aos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= g.nx) return;
    const long long n = (long long)j * g.nx + i;
#pragma unroll
    for (int q = 0; q < 9; ++q) aos[9 * n + q] = soa[q * g.qstride + (long long)j * g.pitch + i];
}

inline int grid1(int N) { return (N + OPS_BLOCK - 1) / OPS_BLOCK; }
inline int ok() { return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH; }

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_feq(const double* ro, const double* U, int N, int incomp, double* feq, void* s)
{
    if (!ro || !U || !feq || N < 0) return IBLBM_E_ARG;
    if (N == 0) return IBLBM_OK;
    feq_kernel<<<grid1(N), OPS_BLOCK, 0, (cudaStream_t)s>>>(ro, U, N, incomp, feq);
    return ok();
}

extern "C" int iblbm_macroscopic(const double* f, int N, int incomp, double* ro, double* U, void* s)
{
    if (!f || !ro || !U || N < 0) return IBLBM_E_ARG;
    if (N == 0) return IBLBM_OK;
    macro_kernel<<<grid1(N), OPS_BLOCK, 0, (cudaStream_t)s>>>(f, N, incomp, ro, U);
    return ok();
}

extern "C" int iblbm_collision_bgk(const double* fs, const double* feq, const double* U, const double* fib, int N,
                                   double tau, double dt, double* f, void* s)
{
    if (!fs || !feq || !U || !fib || !f || N < 0 || !(tau > 0.0)) return IBLBM_E_ARG;
    if (N == 0) return IBLBM_OK;
    bgk_kernel<<<grid1(N), OPS_BLOCK, 0, (cudaStream_t)s>>>(fs, feq, U, fib, N, 1.0 / tau, 1.0 - 0.5 / tau, dt, f);
    return ok();
}

extern "C" int iblbm_collision_trt(const double* fs, const double* feq, const double* U, const double* fib, int N,
                                   double tau, double tau_minus, double dt, double* f, void* s)
{
    if (!fs || !feq || !U || !fib || !f || N < 0 || !(tau > 0.0) || !(tau_minus > 0.0)) return IBLBM_E_ARG;
    if (N == 0) return IBLBM_OK;
    trt_kernel<<<grid1(N), OPS_BLOCK, 0, (cudaStream_t)s>>>(fs, feq, U, fib, N, 1.0 / tau, 1.0 / tau_minus, dt, f);
    return ok();
}

extern "C" int iblbm_collision_cm_mrt(const double* fs, const double* U, const double* fib, int N,
                                      const double* S_diag_host, double dt, double* f, void* s)
{
    if (!fs || !U || !fib || !f || !S_diag_host || N < 0) return IBLBM_E_ARG;
    if (N == 0) return IBLBM_OK;
    S9 S;
    for (int m = 0; m < 9; ++m) S.s[m] = S_diag_host[m];
    cmmrt_kernel<<<grid1(N), OPS_BLOCK, 0, (cudaStream_t)s>>>(fs, U, fib, N, S, dt, f);
    return ok();
}

extern "C" int iblbm_streaming(const double* fold, const double* f, int nx, int ny, double* fnew, void* s)
{
    if (!fold || !f || !fnew || nx < 1 || ny < 1) return IBLBM_E_ARG;
    dim3 grid((nx + 127) / 128, ny);
    stream_kernel<<<grid, 128, 0, (cudaStream_t)s>>>(fold, f, nx, ny, fnew);
    return ok();
}

extern "C" int iblbm_velocity_correction(double* U, const double* fib, const double* ro, int N, double dt, int incomp,
                                         void* s)
{
    if (!U || !fib || !ro || N < 0) return IBLBM_E_ARG;
    if (N == 0) return IBLBM_OK;
    vcorr_kernel<<<grid1(N), OPS_BLOCK, 0, (cudaStream_t)s>>>(U, fib, ro, N, dt, incomp);
    return ok();
}

extern "C" int iblbm_aos_to_soa(const double* aos, iblbm_geom g, double* soa, void* s)
{
    if (!aos || !soa || g.nx < 1 || g.ny < 1 || g.pitch < g.nx) return IBLBM_E_ARG;
    dim3 grid((g.nx + 127) / 128, g.ny);
    aos_to_soa_kernel<<<grid, 128, 0, (cudaStream_t)s>>>(aos, Geom{g.nx, g.ny, g.pitch, g.qstride}, soa);
    return ok();
}

extern "C" int iblbm_soa_to_aos(const double* soa, iblbm_geom g, double* aos, void* s)
{
    if (!aos || !soa || g.nx < 1 || g.ny < 1 || g.pitch < g.nx) return IBLBM_E_ARG;
    dim3 grid((g.nx + 127) / 128, g.ny);
    soa_to_aos_kernel<<<grid, 128, 0, (cudaStream_t)s>>>(soa, Geom{g.nx, g.ny, g.pitch, g.qstride}, aos);
    return ok();
}
