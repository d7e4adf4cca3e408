// common.cuh — D2Q9 lattice constants, lattice geometry and the per-node device
// functions shared by the dense collide-stream kernel and the IBM band kernel.
//
// FP64 "plain" arithmetic contract: every function evaluates the same expression
// tree in the same order as the reference CPU path (numba/numpy, no FMA), and the
// translation units that include this header are compiled with -fmad=false, so
// results are bit-identical to the reference.  Multiplications by lattice vector
// components e in {0, +-1} are exact and written as the adds/subtracts they are.
#pragma once
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>
#include "../../include/iblbm_b200.h"

namespace iblbm {

// Raises kernel K's dynamic shared-memory limit to bytes, once per process and
// thread-safe; later calls return the first call's result.
template <auto K>
inline cudaError_t smem_limit_once(int bytes)
{
    static std::once_flag flag;
    static cudaError_t err = cudaSuccess;
    std::call_once(flag, [&] { err = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes); });
    return err;
}

// D2Q9 ordering of iblbm/lbm/lattice.py:45-55: 0; E,N,W,S; NE,NW,SW,SE
__host__ __device__ constexpr int ex_(int q) { return q == 1 || q == 5 || q == 8 ? 1 : (q == 3 || q == 6 || q == 7 ? -1 : 0); }
__host__ __device__ constexpr int ey_(int q) { return q == 2 || q == 5 || q == 6 ? 1 : (q == 4 || q == 7 || q == 8 ? -1 : 0); }
__host__ __device__ constexpr int opp_(int q) { return q == 0 ? 0 : (q <= 4 ? ((q + 1) % 4 + 1) : ((q - 5 + 2) % 4 + 5)); }
__host__ __device__ constexpr double w_(int q) { return q == 0 ? 4.0 / 9.0 : (q <= 4 ? 1.0 / 9.0 : 1.0 / 36.0); }

enum Collision : int { COLL_BGK = 0, COLL_TRT = 1, COLL_CMMRT = 2 };
enum Boundary : int { BC_DIRICHLET_NEUMANN = 0, BC_OPEN = 1, BC_SETTLING = 2, BC_VELOCITY_INLET = 3, BC_TG = 4 };
enum IbmMethod : int { IBM_NONE = 0, IBM_DF = 1, IBM_MDF = 2, IBM_DFC = 3 };

// Lattice geometry in HBM: one structure-of-arrays plane per population q,
// rows padded to `pitch` elements (a multiple of 32) so every row starts on a
// 256-byte boundary.  Element (q, j, i) lives at q*qstride + j*pitch + i.
struct Geom {
    int nx, ny, pitch;
    long long qstride;  // pitch * ny
};

// Collision parameters (host-computed with the reference's formulas).
struct CollParams {
    double tau, inv_tau, guo_pref;  // BGK: 1/tau, 1 - 0.5/tau   (bgk.py:28-29)
    double s_plus, s_minus;          // TRT: 1/tau, 1/tau_minus  (trt.py:80-86)
    double S[9];                     // CM-MRT relaxation rates  (cm_mrt.py:171-188)
    double dt;
};

struct BcParams {
    int type;
    double inflow_u, dens;
    double feq_in[9];  // feq(dens, (inflow_u, 0)) for the Dirichlet faces
    const double* tg_face;   // Taylor-Green: boundary-node velocities before decay
    const double* tg_decay;  // Taylor-Green: decay factor of this step (device scalar)
};

// Closure constants of a case; feq(dens, (u_in, 0)) in the operation order of
// iblbm/lbm/equilibrium.py:39-42.  Host and device evaluate the same IEEE
// expression (no contraction: x86-64 host code has no FMA, device units are
// compiled with -fmad=false), so both give the same bits.
__host__ __device__ inline void make_bc(const iblbm_case& c, BcParams& bc)
{
    bc.type = c.bc;
    bc.inflow_u = c.inflow_u;
    bc.dens = c.dens;
    bc.tg_face = c.tg_face;
    bc.tg_decay = c.tg_decay;
    const double u0 = c.inflow_u, u1 = 0.0, u2 = u0 * u0 + u1 * u1;
    for (int q = 0; q < 9; ++q) {
        const double a0 = (double)ex_(q) * u0, a1 = (double)ey_(q) * u1, eU = a0 + a1;
        bc.feq_in[q] = c.dens * w_(q) * (1.0 + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
    }
}

// Slot of boundary node (i, j) in the Taylor-Green face table: left j, right j,
// bottom i-1, top i-1, then the corners (0,0), (nx-1,0), (0,ny-1), (nx-1,ny-1).
__host__ __device__ __forceinline__ int tg_slot(int nx, int ny, int i, int j)
{
    if ((i == 0 || i == nx - 1) && (j == 0 || j == ny - 1))
        return 2 * ny + 2 * (nx - 2) + (i == 0 ? 0 : 1) + (j == 0 ? 0 : 2);
    if (i == 0) return j;
    if (i == nx - 1) return ny + j;
    if (j == 0) return 2 * ny + (i - 1);
    return 2 * ny + (nx - 2) + (i - 1);
}

// ---------------------------------------------------------------------------
// Equilibrium — iblbm/lbm/equilibrium.py:27-43
// ---------------------------------------------------------------------------
__device__ __forceinline__ double e_dot(int q, double u0, double u1)
{
    const double a = (double)ex_(q) * u0;
    const double b = (double)ey_(q) * u1;
    return a + b;
}

template <bool INCOMP>
__device__ __forceinline__ double feq_q(int q, double ro, double u0, double u1, double u2)
{
    const double eU = e_dot(q, u0, u1);
    if (INCOMP)
        return w_(q) * (ro + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
    return ro * w_(q) * (1.0 + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
}

__device__ __forceinline__ void feq_all(double ro, double u0, double u1, bool incomp, double* out)
{
    const double u2 = u0 * u0 + u1 * u1;
#pragma unroll
    for (int q = 0; q < 9; ++q)
        out[q] = incomp ? feq_q<true>(q, ro, u0, u1, u2) : feq_q<false>(q, ro, u0, u1, u2);
}

// ---------------------------------------------------------------------------
// Macroscopic — iblbm/lbm/macroscopic.py:27-49 (sequential i = 0..8)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void macro_seq(const double* f, bool incomp, double& ro, double& u0, double& u1)
{
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) s += f[q];
    // ux accumulates f*e_x for q = 0..8; the zero terms leave the sum unchanged
    const double ux = ((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8];
    const double uy = ((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8];
    ro = s;
    if (incomp) { u0 = ux; u1 = uy; }
    else { u0 = ux / s; u1 = uy / s; }
}

// numpy row sum of 9 entries: ((a0+a1)+(a2+a3))+((a4+a5)+(a6+a7)) + a8
__device__ __forceinline__ double np_sum9(double a0, double a1, double a2, double a3, double a4,
                                          double a5, double a6, double a7, double a8)
{
    const double r = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    return r + a8;
}

// _macro_from_streamed — iblbm/boundary/dirichlet_neumann.py:63-69
__device__ __forceinline__ void macro_np(const double* f, double& ro, double& u0, double& u1)
{
    const double r = np_sum9(f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8]);
    // f*e_x row: [0*f0, f1, 0*f2, -f3, 0*f4, f5, -f6, -f7, f8]
    const double z = 0.0;
    const double sx = np_sum9(z * f[0], f[1], z * f[2], -f[3], z * f[4], f[5], -f[6], -f[7], f[8]);
    const double sy = np_sum9(z * f[0], z * f[1], f[2], z * f[3], -f[4], f[5], f[6], -f[7], -f[8]);
    ro = r;
    u0 = sx / r;
    u1 = sy / r;
}

// ---------------------------------------------------------------------------
// Pull streaming — iblbm/lbm/streaming.py:38-77.  A population whose source lies
// outside the lattice is left at 0: every such entry is overwritten by the
// boundary closure of that node before anything reads it.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void pull(const T* __restrict__ fpost, const Geom& g, int i, int j, T* f)
{
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int si = i - ex_(q), sj = j - ey_(q);
        const bool in = (si >= 0) & (si < g.nx) & (sj >= 0) & (sj < g.ny);
        f[q] = in ? fpost[q * g.qstride + (long long)sj * g.pitch + si] : T(0);
    }
}

// Old velocity ring: U of the previous step (after the IBM correction) at the
// rows/columns 1, 2, n-3, n-2 that the extrapolating closures read.
__device__ __forceinline__ double uo_x(const double* __restrict__ ur, const Geom& g, int i, int j)
{
    return ur[2 * ((long long)j * g.nx + i)];
}
__device__ __forceinline__ double uo_y(const double* __restrict__ ur, const Geom& g, int i, int j)
{
    return ur[2 * ((long long)j * g.nx + i) + 1];
}

__device__ __forceinline__ bool is_ring(const Geom& g, int i, int j)
{
    return i == 1 || i == 2 || i == g.nx - 3 || i == g.nx - 2 || j == 1 || j == 2 || j == g.ny - 3 ||
           j == g.ny - 2;
}

// ---------------------------------------------------------------------------
// Boundary closures for one boundary node (i, j): f holds its pulled
// populations on entry and the post-closure populations on exit.
// ---------------------------------------------------------------------------

// iblbm/boundary/dirichlet_neumann.py:39-120
__device__ __forceinline__ void bc_dirichlet_neumann(const double* __restrict__ fpost, const Geom& g,
                                                     const BcParams& bc, int i, int j, double* f)
{
    if (i == g.nx - 1) {
        const int js = (j == 0) ? 1 : (j == g.ny - 1 ? g.ny - 2 : j);
        double fi[9], fq[9], r, a, b;
        pull(fpost, g, g.nx - 2, js, fi);
        macro_np(fi, r, a, b);
        feq_all(r, a, b, false, fq);
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = fq[q] + (fi[q] - fq[q]);
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = bc.feq_in[q];
    }
}

// iblbm/boundary/open_boundary.py:44-165
__device__ __forceinline__ void bc_open(const double* __restrict__ ur, const Geom& g, const BcParams& bc,
                                        int i, int j, double* f)
{
    const int nx = g.nx, ny = g.ny;
    const bool corner = (i == 0 || i == nx - 1) && (j == 0 || j == ny - 1);
    const double ro = bc.dens;
    if (corner) {
        const int di = (i == 0) ? 1 : nx - 2, dj = (j == 0) ? 1 : ny - 2;
        feq_all(ro, uo_x(ur, g, di, dj), uo_y(ur, g, di, dj), false, f);
        return;
    }
    if (i == 0) {
        const double ux = 1.0 - (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[7] + f[6])) / ro;
        const double uy = (4.0 * uo_y(ur, g, 1, j) - uo_y(ur, g, 2, j)) / 3.0;
        f[1] = f[3] + (2.0 / 3.0) * ro * ux;
        f[5] = (f[7] - 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * ro * ux + 0.5 * ro * uy);
        f[8] = (f[6] + 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * ro * ux - 0.5 * ro * uy);
    } else if (i == nx - 1) {
        const double ux = -1.0 + (f[0] + f[2] + f[4] + 2.0 * (f[1] + f[5] + f[8])) / ro;
        const double uy = (4.0 * uo_y(ur, g, nx - 2, j) - uo_y(ur, g, nx - 3, j)) / 3.0;
        f[3] = f[1] - (2.0 / 3.0) * ro * ux;
        f[7] = (f[5] + 0.5 * (f[2] - f[4]) - (1.0 / 6.0) * ro * ux - 0.5 * ro * uy);
        f[6] = (f[8] - 0.5 * (f[2] - f[4]) - (1.0 / 6.0) * ro * ux + 0.5 * ro * uy);
    } else if (j == ny - 1) {
        const double uy = -1.0 + (f[0] + f[1] + f[3] + 2.0 * (f[2] + f[5] + f[6])) / ro;
        const double ux = (4.0 * uo_x(ur, g, i, ny - 2) - uo_x(ur, g, i, ny - 3)) / 3.0;
        f[4] = f[2] - (2.0 / 3.0) * ro * uy;
        f[7] = (f[5] + 0.5 * (f[1] - f[3]) - (1.0 / 6.0) * ro * uy - 0.5 * ro * ux);
        f[8] = (f[6] - 0.5 * (f[1] - f[3]) - (1.0 / 6.0) * ro * uy + 0.5 * ro * ux);
    } else {  // j == 0
        const double uy = 1.0 - (f[0] + f[1] + f[3] + 2.0 * (f[4] + f[7] + f[8])) / ro;
        const double ux = (4.0 * uo_x(ur, g, i, 1) - uo_x(ur, g, i, 2)) / 3.0;
        f[2] = f[4] + (2.0 / 3.0) * ro * uy;
        f[5] = (f[7] - 0.5 * (f[1] - f[3]) + (1.0 / 6.0) * ro * uy + 0.5 * ro * ux);
        f[6] = (f[8] + 0.5 * (f[1] - f[3]) + (1.0 / 6.0) * ro * uy - 0.5 * ro * ux);
    }
}

// iblbm/boundary/settling_channel.py:42-145
__device__ __forceinline__ void bc_settling(const Geom& g, const BcParams& bc, bool incomp, int i, int j,
                                            double* f)
{
    const int nx = g.nx, ny = g.ny;
    if ((i == 0 || i == nx - 1) && (j == 0 || j == ny - 1)) {
        feq_all(bc.dens, 0.0, 0.0, incomp, f);
        return;
    }
    if (i == 0) {
        f[1] = f[3];
        f[5] = (f[7] - 0.5 * (f[2] - f[4]));
        f[8] = (f[6] + 0.5 * (f[2] - f[4]));
    } else if (i == nx - 1) {
        f[3] = f[1];
        f[7] = (f[5] + 0.5 * (f[2] - f[4]));
        f[6] = (f[8] - 0.5 * (f[2] - f[4]));
    } else if (j == ny - 1) {
        f[4] = f[2];
        f[7] = (f[5] + 0.5 * (f[1] - f[3]));
        f[8] = (f[6] - 0.5 * (f[1] - f[3]));
    } else {
        f[2] = f[4];
        f[5] = (f[7] - 0.5 * (f[1] - f[3]));
        f[6] = (f[8] + 0.5 * (f[1] - f[3]));
    }
}

// iblbm/boundary/velocity_inlet.py:45-160 (left/right faces include the corners)
__device__ __forceinline__ void bc_velocity_inlet(const double* __restrict__ ur, const Geom& g,
                                                  const BcParams& bc, int i, int j, double* f)
{
    const int nx = g.nx, ny = g.ny;
    if (i == 0) {
        if (j == 0 || j == ny - 1) {
            feq_all(bc.dens, bc.inflow_u, 0.0, false, f);
            return;
        }
        const double ux = bc.inflow_u, uy = 0.0;
        const double ro = (1.0 / (1.0 - ux)) * (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7]));
        f[1] = f[3] + (2.0 / 3.0) * ro * ux;
        f[5] = (f[7] - 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * ro * ux + 0.5 * ro * uy);
        f[8] = (f[6] + 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * ro * ux - 0.5 * ro * uy);
        return;
    }
    if (i == nx - 1) {
        if (j == 0 || j == ny - 1) {
            // outlet corner: U_x extrapolated from the two neighbouring face nodes,
            // whose U_x this same closure has just extrapolated from the old field
            const int r1 = (j == 0) ? 1 : ny - 2, r2 = (j == 0) ? 2 : ny - 3;
            const double b1 = (4.0 * uo_x(ur, g, nx - 2, r1) - uo_x(ur, g, nx - 2, r2)) / 3.0;
            const double b2 = (4.0 * uo_x(ur, g, nx - 3, r1) - uo_x(ur, g, nx - 3, r2)) / 3.0;
            const double uxc = (4.0 * b1 - b2) / 3.0;
            feq_all(bc.dens, uxc, 0.0, false, f);
            return;
        }
        const double ro = bc.dens;
        const double uy = (4.0 * uo_y(ur, g, nx - 2, j) - uo_y(ur, g, nx - 3, j)) / 3.0;
        const double ux = -1.0 + (f[0] + f[2] + f[4] + 2.0 * (f[1] + f[5] + f[8])) / ro;
        f[3] = f[1] - (2.0 / 3.0) * ro * ux;
        f[7] = (f[5] + 0.5 * (f[2] - f[4]) - (1.0 / 6.0) * ro * ux - 0.5 * ro * uy);
        f[6] = (f[8] - 0.5 * (f[2] - f[4]) - (1.0 / 6.0) * ro * ux + 0.5 * ro * uy);
        return;
    }
    if (j == ny - 1) {
        const double ux = (4.0 * uo_x(ur, g, i, ny - 2) - uo_x(ur, g, i, ny - 3)) / 3.0;
        const double uy = 0.0;
        const double ro = (1.0 / (1.0 + uy)) * (f[0] + f[1] + f[3] + 2.0 * (f[2] + f[5] + f[6]));
        f[4] = f[2] - (2.0 / 3.0) * ro * uy;
        f[7] = (f[5] + 0.5 * (f[1] - f[3]) - 0.5 * ro * ux);
        f[8] = (f[6] - 0.5 * (f[1] - f[3]) + 0.5 * ro * ux);
        return;
    }
    {  // j == 0
        const double ux = (4.0 * uo_x(ur, g, i, 1) - uo_x(ur, g, i, 2)) / 3.0;
        const double uy = 0.0;
        const double ro = (1.0 / (1.0 - uy)) * (f[0] + f[1] + f[3] + 2.0 * (f[4] + f[7] + f[8]));
        f[2] = f[4] + (2.0 / 3.0) * ro * uy;
        f[5] = (f[7] - 0.5 * (f[1] - f[3]) + 0.5 * ro * ux);
        f[6] = (f[8] + 0.5 * (f[1] - f[3]) - 0.5 * ro * ux);
    }
}

// iblbm/boundary/tg_analytical.py:26-170: the analytic velocity u imposed on all
// four faces by Zou-He closures, the corners reset to feq(1, u); u is the node's
// tabulated velocity times this step's decay factor (the reference's
// ((-u0 cos) sin) * decay with the same rounding).
__device__ __forceinline__ void bc_tg(const Geom& g, const BcParams& bc, int i, int j, double* f)
{
    const int nx = g.nx, ny = g.ny;
    const int k = tg_slot(nx, ny, i, j);
    const double d = *bc.tg_decay;
    const double ux = bc.tg_face[2 * k] * d, uy = bc.tg_face[2 * k + 1] * d;
    if ((i == 0 || i == nx - 1) && (j == 0 || j == ny - 1)) {
        feq_all(1.0, ux, uy, false, f);
        return;
    }
    if (i == 0) {
        const double ro = (1.0 / (1.0 - ux)) * (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7]));
        f[1] = f[3] + (2.0 / 3.0) * ro * ux;
        f[5] = (f[7] - 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * ro * ux + 0.5 * ro * uy);
        f[8] = (f[6] + 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * ro * ux - 0.5 * ro * uy);
    } else if (i == nx - 1) {
        const double ro = (1.0 / (1.0 + ux)) * (f[0] + f[2] + f[4] + 2.0 * (f[1] + f[5] + f[8]));
        f[3] = f[1] - (2.0 / 3.0) * ro * ux;
        f[7] = (f[5] + 0.5 * (f[2] - f[4]) - (1.0 / 6.0) * ro * ux - 0.5 * ro * uy);
        f[6] = (f[8] - 0.5 * (f[2] - f[4]) - (1.0 / 6.0) * ro * ux + 0.5 * ro * uy);
    } else if (j == ny - 1) {
        const double ro = (1.0 / (1.0 + uy)) * (f[0] + f[1] + f[3] + 2.0 * (f[2] + f[5] + f[6]));
        f[4] = f[2] - (2.0 / 3.0) * ro * uy;
        f[7] = (f[5] + 0.5 * (f[1] - f[3]) - (1.0 / 6.0) * ro * uy - 0.5 * ro * ux);
        f[8] = (f[6] - 0.5 * (f[1] - f[3]) - (1.0 / 6.0) * ro * uy + 0.5 * ro * ux);
    } else {  // j == 0
        const double ro = (1.0 / (1.0 - uy)) * (f[0] + f[1] + f[3] + 2.0 * (f[4] + f[7] + f[8]));
        f[2] = f[4] + (2.0 / 3.0) * ro * uy;
        f[5] = (f[7] - 0.5 * (f[1] - f[3]) + (1.0 / 6.0) * ro * uy + 0.5 * ro * ux);
        f[6] = (f[8] + 0.5 * (f[1] - f[3]) + (1.0 / 6.0) * ro * uy - 0.5 * ro * ux);
    }
}

// Post-streaming, post-closure populations of node (i, j) — iblbm/runtime/step.py:49-60
// (streaming_step then apply_boundary_step).
template <int BC>
__device__ __forceinline__ void fstar_node(const double* __restrict__ fpost, const double* __restrict__ ur,
                                           const Geom& g, const BcParams& bc, bool incomp, int i, int j,
                                           double* f)
{
    const bool boundary = (i == 0) | (j == 0) | (i == g.nx - 1) | (j == g.ny - 1);
    if (BC == BC_DIRICHLET_NEUMANN && boundary) {
        bc_dirichlet_neumann(fpost, g, bc, i, j, f);
        return;
    }
    pull(fpost, g, i, j, f);
    if (!boundary) return;
    if (BC == BC_OPEN) bc_open(ur, g, bc, i, j, f);
    else if (BC == BC_SETTLING) bc_settling(g, bc, incomp, i, j, f);
    else if (BC == BC_VELOCITY_INLET) bc_velocity_inlet(ur, g, bc, i, j, f);
    else if (BC == BC_TG) bc_tg(g, bc, i, j, f);
}

// ---------------------------------------------------------------------------
// Immersed-boundary delta kernels — iblbm/ibm/common.py:52-119
// ---------------------------------------------------------------------------
__device__ __forceinline__ double phi_hat(double r)
{
    const double v = 1.0 - fabs(r);
    return v > 0.0 ? v : 0.0;
}

__device__ __forceinline__ double phi_p4(double r)
{
    const double ar = fabs(r);
    if (ar <= 1.0) {
        double s = 1.0 + 4.0 * ar - 4.0 * (ar * ar);
        s = s > 0.0 ? s : 0.0;
        return (1.0 / 8.0) * (3.0 - 2.0 * ar + sqrt(s));
    }
    if (ar <= 2.0) {
        double s = -7.0 + 12.0 * ar - 4.0 * (ar * ar);
        s = s > 0.0 ? s : 0.0;
        return (1.0 / 8.0) * (5.0 - 2.0 * ar - sqrt(s));
    }
    return 0.0;
}

// delta type ids: 0 = peskin4pt (radius 2), 1 = hat (radius 1)
__device__ __forceinline__ double phi(int delta_type, double r) { return delta_type == 0 ? phi_p4(r) : phi_hat(r); }

}  // namespace iblbm
