// shifted.cuh — FP32 "shifted population" form of the per-node timestep.
//
// Populations are stored and collided as deviations g_q = f_q - w_q in FP32.
// The O(1) lattice weights never enter an FP32 sum, so the deviations keep
// ~7 significant digits of the O(u) physics instead of losing 2-3 digits to
// cancellation against w_q.  Identities used (lattice weights w_q = w_opp(q),
// sum w = 1, sum w e = 0, sum w e_x^2 = 1/3, sum w e_x^2 e_y^2 = 1/9):
//   rho = 1 + sum g,  rho u = sum g e;
//   feq_q - w_q = w_q (d_rho + rho X_q)          (compressible)
//              = w_q (d_rho + X_q)              (incompressible, He-Luo)
//   with X_q = 3 e.u + 4.5 (e.u)^2 - 1.5 u^2 and d_rho = rho - 1;
//   the Zou-He unknown-population formulas pair equal weights, so they hold
//   unchanged on g, and their density sums become 1 + (sum of the g's);
//   CM-MRT relaxes k(g) with the analytic central moments of the weights
//   k(w) about u, and maps the post-collision difference back with the same
//   linear transform, so g_out = T(k_post - k(w)).
// Arithmetic is FP32 (contracted to FMA where the compiler chooses).
#pragma once
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

struct BcParams32 {
    float inflow_u, dens;
    float geq_in[9];  // feq(dens, (inflow_u, 0)) - w, rounded from FP64
    const double* tg_face;   // Taylor-Green: boundary-node velocities before decay (FP64)
    const double* tg_decay;  // Taylor-Green: decay factor of this step (device scalar)
};

struct CollParams32 {
    float inv_tau, guo_pref, s_plus, s_minus, dt;
    float S[9];
};

// Closure constants of a case, rounded from its FP64 parameters.
__host__ __device__ inline void make_bc(const iblbm_case& c, BcParams32& bc)
{
    bc.inflow_u = (float)c.inflow_u;
    bc.dens = (float)c.dens;
    bc.tg_face = c.tg_face;
    bc.tg_decay = c.tg_decay;
    const double u0 = c.inflow_u, u2 = u0 * u0;
    for (int q = 0; q < 9; ++q) {
        const double eU = (double)ex_(q) * u0;
        const double feq = c.dens * w_(q) * (1.0 + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
        bc.geq_in[q] = (float)(feq - w_(q));
    }
}

__device__ __forceinline__ float wf(int q) { return (float)w_(q); }

// feq - w in shifted form
template <bool INCOMP>
__device__ __forceinline__ float geq_q(int q, float drho, float rho, float u0, float u1, float u2)
{
    const float eu = (float)ex_(q) * u0 + (float)ey_(q) * u1;
    const float X = 3.0f * eu + 4.5f * eu * eu - 1.5f * u2;
    return INCOMP ? wf(q) * (drho + X) : wf(q) * (drho + rho * X);
}

__device__ __forceinline__ void macro_g(const float* g, bool incomp, float& drho, float& rho, float& u0, float& u1)
{
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 9; ++q) s += g[q];
    const float jx = ((g[1] - g[3]) + (g[5] - g[6])) + (g[8] - g[7]);
    const float jy = ((g[2] - g[4]) + (g[5] + g[6])) - (g[7] + g[8]);
    drho = s;
    rho = 1.0f + s;
    if (incomp) { u0 = jx; u1 = jy; }
    else { const float inv = 1.0f / rho; u0 = jx * inv; u1 = jy * inv; }
}

__device__ __forceinline__ void geq_all(float dens, float u0, float u1, bool incomp, float* out)
{
    const float drho = dens - 1.0f, u2 = u0 * u0 + u1 * u1;
#pragma unroll
    for (int q = 0; q < 9; ++q) out[q] = incomp ? geq_q<true>(q, drho, dens, u0, u1, u2) : geq_q<false>(q, drho, dens, u0, u1, u2);
}

// ---- boundary closures on g (see the formulas of common.cuh) ---------------------
__device__ __forceinline__ float uo32_x(const float* __restrict__ ur, const Geom& g, int i, int j)
{
    return ur[2 * ((long long)j * g.nx + i)];
}
__device__ __forceinline__ float uo32_y(const float* __restrict__ ur, const Geom& g, int i, int j)
{
    return ur[2 * ((long long)j * g.nx + i) + 1];
}

__device__ __forceinline__ void bc32_dirichlet_neumann(const float* __restrict__ fp, const Geom& g, const BcParams32& bc,
                                                       int i, int j, float* f)
{
    if (i == g.nx - 1) {
        const int js = (j == 0) ? 1 : (j == g.ny - 1 ? g.ny - 2 : j);
        float fi[9], fq[9], drho, rho, a, b;
        pull(fp, g, g.nx - 2, js, fi);
        macro_g(fi, false, drho, rho, a, b);
        geq_all(rho, a, b, false, fq);
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = fq[q] + (fi[q] - fq[q]);
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = bc.geq_in[q];
    }
}

__device__ __forceinline__ void bc32_open(const float* __restrict__ ur, const Geom& g, const BcParams32& bc, int i,
                                          int j, float* f)
{
    const int nx = g.nx, ny = g.ny;
    const float ro = bc.dens, dr = bc.dens - 1.0f;
    if ((i == 0 || i == nx - 1) && (j == 0 || j == ny - 1)) {
        const int di = (i == 0) ? 1 : nx - 2, dj = (j == 0) ? 1 : ny - 2;
        geq_all(ro, uo32_x(ur, g, di, dj), uo32_y(ur, g, di, dj), false, f);
        return;
    }
    if (i == 0) {
        const float G = f[0] + f[2] + f[4] + 2.0f * (f[3] + f[7] + f[6]);
        const float ux = (dr - G) / ro;
        const float uy = (4.0f * uo32_y(ur, g, 1, j) - uo32_y(ur, g, 2, j)) / 3.0f;
        f[1] = f[3] + (2.0f / 3.0f) * ro * ux;
        f[5] = f[7] - 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * ro * ux + 0.5f * ro * uy;
        f[8] = f[6] + 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * ro * ux - 0.5f * ro * uy;
    } else if (i == nx - 1) {
        const float G = f[0] + f[2] + f[4] + 2.0f * (f[1] + f[5] + f[8]);
        const float ux = (G - dr) / ro;
        const float uy = (4.0f * uo32_y(ur, g, nx - 2, j) - uo32_y(ur, g, nx - 3, j)) / 3.0f;
        f[3] = f[1] - (2.0f / 3.0f) * ro * ux;
        f[7] = f[5] + 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * ro * ux - 0.5f * ro * uy;
        f[6] = f[8] - 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * ro * ux + 0.5f * ro * uy;
    } else if (j == ny - 1) {
        const float G = f[0] + f[1] + f[3] + 2.0f * (f[2] + f[5] + f[6]);
        const float uy = (G - dr) / ro;
        const float ux = (4.0f * uo32_x(ur, g, i, ny - 2) - uo32_x(ur, g, i, ny - 3)) / 3.0f;
        f[4] = f[2] - (2.0f / 3.0f) * ro * uy;
        f[7] = f[5] + 0.5f * (f[1] - f[3]) - (1.0f / 6.0f) * ro * uy - 0.5f * ro * ux;
        f[8] = f[6] - 0.5f * (f[1] - f[3]) - (1.0f / 6.0f) * ro * uy + 0.5f * ro * ux;
    } else {
        const float G = f[0] + f[1] + f[3] + 2.0f * (f[4] + f[7] + f[8]);
        const float uy = (dr - G) / ro;
        const float ux = (4.0f * uo32_x(ur, g, i, 1) - uo32_x(ur, g, i, 2)) / 3.0f;
        f[2] = f[4] + (2.0f / 3.0f) * ro * uy;
        f[5] = f[7] - 0.5f * (f[1] - f[3]) + (1.0f / 6.0f) * ro * uy + 0.5f * ro * ux;
        f[6] = f[8] + 0.5f * (f[1] - f[3]) + (1.0f / 6.0f) * ro * uy - 0.5f * ro * ux;
    }
}

__device__ __forceinline__ void bc32_settling(const Geom& g, const BcParams32& bc, bool incomp, int i, int j, float* f)
{
    const int nx = g.nx, ny = g.ny;
    if ((i == 0 || i == nx - 1) && (j == 0 || j == ny - 1)) {
        geq_all(bc.dens, 0.0f, 0.0f, incomp, f);
        return;
    }
    if (i == 0) {
        f[1] = f[3];
        f[5] = f[7] - 0.5f * (f[2] - f[4]);
        f[8] = f[6] + 0.5f * (f[2] - f[4]);
    } else if (i == nx - 1) {
        f[3] = f[1];
        f[7] = f[5] + 0.5f * (f[2] - f[4]);
        f[6] = f[8] - 0.5f * (f[2] - f[4]);
    } else if (j == ny - 1) {
        f[4] = f[2];
        f[7] = f[5] + 0.5f * (f[1] - f[3]);
        f[8] = f[6] - 0.5f * (f[1] - f[3]);
    } else {
        f[2] = f[4];
        f[5] = f[7] - 0.5f * (f[1] - f[3]);
        f[6] = f[8] + 0.5f * (f[1] - f[3]);
    }
}

__device__ __forceinline__ void bc32_velocity_inlet(const float* __restrict__ ur, const Geom& g, const BcParams32& bc,
                                                    int i, int j, float* f)
{
    const int nx = g.nx, ny = g.ny;
    if (i == 0) {
        if (j == 0 || j == ny - 1) {
            geq_all(bc.dens, bc.inflow_u, 0.0f, false, f);
            return;
        }
        const float ux = bc.inflow_u, uy = 0.0f;
        const float ro = (1.0f + (f[0] + f[2] + f[4] + 2.0f * (f[3] + f[6] + f[7]))) / (1.0f - ux);
        f[1] = f[3] + (2.0f / 3.0f) * ro * ux;
        f[5] = f[7] - 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * ro * ux + 0.5f * ro * uy;
        f[8] = f[6] + 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * ro * ux - 0.5f * ro * uy;
        return;
    }
    if (i == nx - 1) {
        if (j == 0 || j == ny - 1) {
            const int r1 = (j == 0) ? 1 : ny - 2, r2 = (j == 0) ? 2 : ny - 3;
            const float b1 = (4.0f * uo32_x(ur, g, nx - 2, r1) - uo32_x(ur, g, nx - 2, r2)) / 3.0f;
            const float b2 = (4.0f * uo32_x(ur, g, nx - 3, r1) - uo32_x(ur, g, nx - 3, r2)) / 3.0f;
            geq_all(bc.dens, (4.0f * b1 - b2) / 3.0f, 0.0f, false, f);
            return;
        }
        const float ro = bc.dens, dr = bc.dens - 1.0f;
        const float uy = (4.0f * uo32_y(ur, g, nx - 2, j) - uo32_y(ur, g, nx - 3, j)) / 3.0f;
        const float ux = ((f[0] + f[2] + f[4] + 2.0f * (f[1] + f[5] + f[8])) - dr) / ro;
        f[3] = f[1] - (2.0f / 3.0f) * ro * ux;
        f[7] = f[5] + 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * ro * ux - 0.5f * ro * uy;
        f[6] = f[8] - 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * ro * ux + 0.5f * ro * uy;
        return;
    }
    if (j == ny - 1) {
        const float ux = (4.0f * uo32_x(ur, g, i, ny - 2) - uo32_x(ur, g, i, ny - 3)) / 3.0f;
        const float ro = 1.0f + (f[0] + f[1] + f[3] + 2.0f * (f[2] + f[5] + f[6]));
        f[4] = f[2];
        f[7] = f[5] + 0.5f * (f[1] - f[3]) - 0.5f * ro * ux;
        f[8] = f[6] - 0.5f * (f[1] - f[3]) + 0.5f * ro * ux;
        return;
    }
    const float ux = (4.0f * uo32_x(ur, g, i, 1) - uo32_x(ur, g, i, 2)) / 3.0f;
    const float ro = 1.0f + (f[0] + f[1] + f[3] + 2.0f * (f[4] + f[7] + f[8]));
    f[2] = f[4];
    f[5] = f[7] - 0.5f * (f[1] - f[3]) + 0.5f * ro * ux;
    f[6] = f[8] + 0.5f * (f[1] - f[3]) - 0.5f * ro * ux;
}

// Taylor-Green faces on g = f - w (iblbm/boundary/tg_analytical.py:26-170): the
// weights of the known populations of a face sum to 1, so rho = (1 + G) / (1 -+ u)
// with G their sum in g, and the unknowns keep the form of the closure on f.
__device__ __forceinline__ void bc32_tg(const Geom& g, const BcParams32& bc, int i, int j, float* f)
{
    const int nx = g.nx, ny = g.ny;
    const int k = tg_slot(nx, ny, i, j);
    const double d = *bc.tg_decay;
    const float ux = (float)(bc.tg_face[2 * k] * d), uy = (float)(bc.tg_face[2 * k + 1] * d);
    if ((i == 0 || i == nx - 1) && (j == 0 || j == ny - 1)) {
        geq_all(1.0f, ux, uy, false, f);
        return;
    }
    if (i == 0) {
        const float ro = (1.0f + (f[0] + f[2] + f[4] + 2.0f * (f[3] + f[6] + f[7]))) / (1.0f - ux);
        f[1] = f[3] + (2.0f / 3.0f) * ro * ux;
        f[5] = f[7] - 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * ro * ux + 0.5f * ro * uy;
        f[8] = f[6] + 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * ro * ux - 0.5f * ro * uy;
    } else if (i == nx - 1) {
        const float ro = (1.0f + (f[0] + f[2] + f[4] + 2.0f * (f[1] + f[5] + f[8]))) / (1.0f + ux);
        f[3] = f[1] - (2.0f / 3.0f) * ro * ux;
        f[7] = f[5] + 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * ro * ux - 0.5f * ro * uy;
        f[6] = f[8] - 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * ro * ux + 0.5f * ro * uy;
    } else if (j == ny - 1) {
        const float ro = (1.0f + (f[0] + f[1] + f[3] + 2.0f * (f[2] + f[5] + f[6]))) / (1.0f + uy);
        f[4] = f[2] - (2.0f / 3.0f) * ro * uy;
        f[7] = f[5] + 0.5f * (f[1] - f[3]) - (1.0f / 6.0f) * ro * uy - 0.5f * ro * ux;
        f[8] = f[6] - 0.5f * (f[1] - f[3]) - (1.0f / 6.0f) * ro * uy + 0.5f * ro * ux;
    } else {
        const float ro = (1.0f + (f[0] + f[1] + f[3] + 2.0f * (f[4] + f[7] + f[8]))) / (1.0f - uy);
        f[2] = f[4] + (2.0f / 3.0f) * ro * uy;
        f[5] = f[7] - 0.5f * (f[1] - f[3]) + (1.0f / 6.0f) * ro * uy + 0.5f * ro * ux;
        f[6] = f[8] + 0.5f * (f[1] - f[3]) + (1.0f / 6.0f) * ro * uy - 0.5f * ro * ux;
    }
}

template <int BC>
__device__ __forceinline__ void gstar_node(const float* __restrict__ fp, const float* __restrict__ ur, const Geom& g,
                                           const BcParams32& bc, bool incomp, int i, int j, float* f)
{
    const bool boundary = (i == 0) | (j == 0) | (i == g.nx - 1) | (j == g.ny - 1);
    if (BC == BC_DIRICHLET_NEUMANN && boundary) {
        bc32_dirichlet_neumann(fp, g, bc, i, j, f);
        return;
    }
    pull(fp, g, i, j, f);
    if (!boundary) return;
    if (BC == BC_OPEN) bc32_open(ur, g, bc, i, j, f);
    else if (BC == BC_SETTLING) bc32_settling(g, bc, incomp, i, j, f);
    else if (BC == BC_VELOCITY_INLET) bc32_velocity_inlet(ur, g, bc, i, j, f);
    else if (BC == BC_TG) bc32_tg(g, bc, i, j, f);
}

// Pull offsets of an interior node relative to its own site: population q
// comes from q*qstride - ey(q)*pitch - ex(q) (fits an int: the host checks
// 9 * qstride < 2^31).
__device__ __forceinline__ void pull_offsets(const Geom& g, int* off)
{
#pragma unroll
    for (int q = 0; q < 9; ++q) off[q] = q * (int)g.qstride - ey_(q) * g.pitch - ex_(q);
}

// Pull of node (i, j): interior nodes read through the precomputed offsets,
// edge nodes through the bounds-checked pull.
__device__ __forceinline__ void pull_node(const float* __restrict__ fp, const Geom& g, const int* off, int i, int j,
                                          float* f)
{
    if (i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) {
        const float* site = fp + (long long)j * g.pitch + i;
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = __ldg(site + off[q]);
    } else {
        pull(fp, g, i, j, f);
    }
}

// Closure of a node whose pulled populations are already in f (the Dirichlet /
// Neumann edge recomputes them from its neighbour column instead).
template <int BC>
__device__ __forceinline__ void closure_node(const float* __restrict__ fp, const float* __restrict__ ur,
                                             const Geom& g, const BcParams32& bc, bool incomp, int i, int j,
                                             float* f)
{
    const bool boundary = (i == 0) | (j == 0) | (i == g.nx - 1) | (j == g.ny - 1);
    if (!boundary) return;
    if (BC == BC_DIRICHLET_NEUMANN) bc32_dirichlet_neumann(fp, g, bc, i, j, f);
    else if (BC == BC_OPEN) bc32_open(ur, g, bc, i, j, f);
    else if (BC == BC_SETTLING) bc32_settling(g, bc, incomp, i, j, f);
    else if (BC == BC_TG) bc32_tg(g, bc, i, j, f);
    else bc32_velocity_inlet(ur, g, bc, i, j, f);
}

// ---- collisions on g ----------------------------------------------------------
__device__ __forceinline__ float guo_bare(int q, float u0, float u1, float F0, float F1)
{
    const float ex = (float)ex_(q), ey = (float)ey_(q);
    const float eU = ex * u0 + ey * u1;
    return wf(q) * ((3.0f * (ex - u0) + 9.0f * eU * ex) * F0 + (3.0f * (ey - u1) + 9.0f * eU * ey) * F1);
}

// The four opposite pairs (q, opp q) with e_q = (+1, 0), (0, +1), (+1, +1), (-1, +1).
__device__ __forceinline__ constexpr int pair_q(int p) { return p == 0 ? 1 : (p == 1 ? 2 : (p == 2 ? 5 : 6)); }

// Equilibrium deviation of a pair, split into its even part (same for q and
// opp q) and odd part (sign flips): geq_q = even + odd, geq_opp = even - odd.
template <bool INCOMP>
__device__ __forceinline__ void geq_pair(int q, float drho, float rho, float u0, float u1, float u2, float& even,
                                         float& odd)
{
    const float eu = (float)ex_(q) * u0 + (float)ey_(q) * u1;
    const float r = INCOMP ? 1.0f : rho;
    even = wf(q) * (drho + r * (4.5f * eu * eu - 1.5f * u2));
    odd = wf(q) * r * 3.0f * eu;
}

template <bool INCOMP, bool FORCED>
__device__ __forceinline__ void collide32_bgk(const float* g, float drho, float rho, float u0, float u1, float F0,
                                              float F1, const CollParams32& cp, float* out)
{
    const float u2 = u0 * u0 + u1 * u1;
    const float fp = cp.guo_pref * cp.dt;
    {
        const float ge = wf(0) * (drho + (INCOMP ? 1.0f : rho) * (-1.5f * u2));
        float v = g[0] - cp.inv_tau * (g[0] - ge);
        if (FORCED) v += fp * guo_bare(0, u0, u1, F0, F1);
        out[0] = v;
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int q = pair_q(p), o = opp_(q);
        float even, odd;
        geq_pair<INCOMP>(q, drho, rho, u0, u1, u2, even, odd);
        float vq = g[q] - cp.inv_tau * (g[q] - (even + odd));
        float vo = g[o] - cp.inv_tau * (g[o] - (even - odd));
        if (FORCED) {
            vq += fp * guo_bare(q, u0, u1, F0, F1);
            vo += fp * guo_bare(o, u0, u1, F0, F1);
        }
        out[q] = vq;
        out[o] = vo;
    }
}

// TRT on pairs: the even part relaxes with s+, the odd part with s-.
template <bool INCOMP, bool FORCED>
__device__ __forceinline__ void collide32_trt(const float* g, float drho, float rho, float u0, float u1, float F0,
                                              float F1, const CollParams32& cp, float* out)
{
    const float u2 = u0 * u0 + u1 * u1;
    const float gp = 1.0f - 0.5f * cp.s_plus, gm = 1.0f - 0.5f * cp.s_minus;
    {
        const float ge = wf(0) * (drho + (INCOMP ? 1.0f : rho) * (-1.5f * u2));
        float v = g[0] - cp.s_plus * (g[0] - ge);
        if (FORCED) v += gp * guo_bare(0, u0, u1, F0, F1) * cp.dt;
        out[0] = v;
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int q = pair_q(p), o = opp_(q);
        float even, odd;
        geq_pair<INCOMP>(q, drho, rho, u0, u1, u2, even, odd);
        const float ne = 0.5f * (g[q] + g[o]) - even;  // non-equilibrium, even part
        const float no = 0.5f * (g[q] - g[o]) - odd;   // non-equilibrium, odd part
        float vq = g[q] - (cp.s_plus * ne + cp.s_minus * no);
        float vo = g[o] - (cp.s_plus * ne - cp.s_minus * no);
        if (FORCED) {
            const float bq = guo_bare(q, u0, u1, F0, F1), bo = guo_bare(o, u0, u1, F0, F1);
            const float be = 0.5f * (bq + bo), bd = 0.5f * (bq - bo);
            vq += (gp * be + gm * bd) * cp.dt;
            vo += (gp * be - gm * bd) * cp.dt;
        }
        out[q] = vq;
        out[o] = vo;
    }
}

// CM-MRT: raw moments of g (sums and differences of populations, e in {0, +-1}),
// shifted to central moments about u by the binomial formulas.  Only the change
// of the central moments, dc = c_post - k(g), is mapped back (the map is
// linear): g_out = g + T(dc), where the conserved moments (m < 3, rate 0) change
// only by the forcing.
template <bool FORCED>
__device__ __forceinline__ void collide32_cmmrt(const float* g, float drho, float ux, float uy, float F0, float F1,
                                                const CollParams32& cp, float* out)
{
    const float s57 = g[5] + g[7], s68 = g[6] + g[8], d57 = g[5] - g[7], d68 = g[6] - g[8];
    const float m00 = (g[0] + (g[1] + g[3])) + ((g[2] + g[4]) + (s57 + s68));
    const float m10 = (g[1] - g[3]) + (d57 - d68);
    const float m01 = (g[2] - g[4]) + (d57 + d68);
    const float m20 = (g[1] + g[3]) + (s57 + s68);
    const float m02 = (g[2] + g[4]) + (s57 + s68);
    const float m11 = s57 - s68;
    const float m21 = d57 + d68;
    const float m12 = d57 - d68;
    const float m22 = s57 + s68;
    const float ux2 = ux * ux, uy2 = uy * uy, uxy = ux * uy;
    float k[9];
    k[3] = m20 - 2.0f * ux * m10 + ux2 * m00;
    k[4] = m02 - 2.0f * uy * m01 + uy2 * m00;
    k[5] = m11 - ux * m01 - uy * m10 + uxy * m00;
    k[6] = m21 - 2.0f * ux * m11 - uy * m20 + ux2 * m01 + 2.0f * uxy * m10 - ux2 * uy * m00;
    k[7] = m12 - 2.0f * uy * m11 - ux * m02 + uy2 * m10 + 2.0f * uxy * m01 - ux * uy2 * m00;
    k[8] = m22 - 2.0f * ux * m12 - 2.0f * uy * m21 + ux2 * m02 + uy2 * m20 + 4.0f * uxy * m11 -
           2.0f * ux * uy2 * m10 - 2.0f * ux2 * uy * m01 + ux2 * uy2 * m00;
    float F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (FORCED) {
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float ex = (float)ex_(q), ey = (float)ey_(q);
            const float cx = ex - ux, cy = ey - uy, cx2 = cx * cx, cy2 = cy * cy;
            const float b = guo_bare(q, ux, uy, F0, F1);
            F[0] += b; F[1] += b * cx; F[2] += b * cy; F[3] += b * cx2; F[4] += b * cy2;
            F[5] += b * cx * cy; F[6] += b * cx2 * cy; F[7] += b * cx * cy2; F[8] += b * cx2 * cy2;
        }
    }
    // central moments of the weights about u, and the equilibrium minus them
    const float ax = 1.0f / 3.0f + ux2, ay = 1.0f / 3.0f + uy2;
    const float rho = 1.0f + drho;
    const float keq3 = rho * (1.0f / 3.0f), keq8 = rho * (1.0f / 9.0f);
    // dc = -S (k(g) + k(w) - k_eq) [+ (1 - S/2) F dt]
    float dc[9];
    dc[3] = -cp.S[3] * (k[3] + (ax - keq3));
    dc[4] = -cp.S[4] * (k[4] + (ay - keq3));
    dc[5] = -cp.S[5] * (k[5] + uxy);
    dc[6] = -cp.S[6] * (k[6] - uy * ax);
    dc[7] = -cp.S[7] * (k[7] - ux * ay);
    dc[8] = -cp.S[8] * (k[8] + (ax * ay - keq8));
    dc[0] = dc[1] = dc[2] = 0.0f;
    if (FORCED) {
#pragma unroll
        for (int m = 0; m < 9; ++m) dc[m] += (1.0f - 0.5f * cp.S[m]) * F[m] * cp.dt;
    }
    // central -> raw moments of the change
    const float K0 = dc[0];
    const float K1 = dc[1] + ux * dc[0];
    const float K2 = dc[2] + uy * dc[0];
    const float K3 = dc[3] + 2.0f * ux * dc[1] + ux2 * dc[0];
    const float K4 = dc[4] + 2.0f * uy * dc[2] + uy2 * dc[0];
    const float K5 = dc[5] + uy * dc[1] + ux * dc[2] + uxy * dc[0];
    const float K6 = dc[6] + uy * dc[3] + 2.0f * ux * dc[5] + 2.0f * uxy * dc[1] + ux2 * dc[2] + ux2 * uy * dc[0];
    const float K7 = dc[7] + 2.0f * uy * dc[5] + ux * dc[4] + 2.0f * uxy * dc[2] + uy2 * dc[1] + ux * uy2 * dc[0];
    const float K8 = dc[8] + 2.0f * uy * dc[6] + uy2 * dc[3] + 2.0f * ux * dc[7] + 4.0f * uxy * dc[5] +
                     2.0f * ux * uy2 * dc[1] + ux2 * dc[4] + 2.0f * ux2 * uy * dc[2] + ux2 * uy2 * dc[0];
    // raw moments -> populations
    out[0] = g[0] + (K0 - K3 - K4 + K8);
    out[1] = g[1] + 0.5f * (K1 + K3 - K7 - K8);
    out[2] = g[2] + 0.5f * (K2 + K4 - K6 - K8);
    out[3] = g[3] + 0.5f * (-K1 + K3 + K7 - K8);
    out[4] = g[4] + 0.5f * (-K2 + K4 + K6 - K8);
    out[5] = g[5] + 0.25f * (K5 + K6 + K7 + K8);
    out[6] = g[6] + 0.25f * (-K5 + K6 - K7 + K8);
    out[7] = g[7] + 0.25f * (K5 - K6 - K7 + K8);
    out[8] = g[8] + 0.25f * (-K5 - K6 + K7 + K8);
}

template <int COLL, bool INCOMP, bool FORCED>
__device__ __forceinline__ void collide32(const float* g, float drho, float rho, float u0, float u1, float F0, float F1,
                                          const CollParams32& cp, float* out)
{
    if (COLL == COLL_BGK) collide32_bgk<INCOMP, FORCED>(g, drho, rho, u0, u1, F0, F1, cp, out);
    else if (COLL == COLL_TRT) collide32_trt<INCOMP, FORCED>(g, drho, rho, u0, u1, F0, F1, cp, out);
    else collide32_cmmrt<FORCED>(g, drho, u0, u1, F0, F1, cp, out);
}

struct BandView32 {
    const int* box;
    const int* map;
    const float* fib;  // band x 2
    const float* df;   // band x 9 (shifted distribution correction)
};

struct DenseOut32 {
    float* fpost_next;
    float* uring_next;
    float* ro_out;
    float* U_out;
    float* fstar_out;
};

__device__ __forceinline__ int band_lookup32(const BandView32& bv, int nx, int i, int j)
{
    const int x0 = __ldg(bv.box + 0), y0 = __ldg(bv.box + 1), w = __ldg(bv.box + 2), h = __ldg(bv.box + 3);
    if (i < x0 || i >= x0 + w || j < y0 || j >= y0 + h) return -1;
    return bv.map[(long long)j * nx + i];
}

// Everything after streaming and closure for node (i, j): band correction,
// optional f* output, moments, velocity correction, collision, ro/U outputs and
// the velocity ring.  f holds the post-streaming populations; out receives the
// post-collision populations (stored by the caller).
template <int COLL, bool RING, bool INCOMP, int IBM, bool OUT>
__device__ __forceinline__ void node_core32(float* f, const Geom& g, const CollParams32& cp,
                                            const BandView32& band, const DenseOut32& o, int i, int j, float* out)
{
    int b = -1;
    if (IBM != IBM_NONE) b = band_lookup32(band, g.nx, i, j);
    if (IBM == IBM_DFC && b >= 0) {
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] += band.df[9 * (long long)b + q];
    }
    const long long site = (long long)j * g.pitch + i;
    if (OUT && o.fstar_out) {
#pragma unroll
        for (int q = 0; q < 9; ++q) o.fstar_out[q * g.qstride + site] = f[q];
    }
    float drho, rho, u0, u1;
    macro_g(f, INCOMP, drho, rho, u0, u1);
    if ((IBM == IBM_DF || IBM == IBM_MDF) && b >= 0) {
        const float F0 = band.fib[2 * (long long)b], F1 = band.fib[2 * (long long)b + 1];
        if (INCOMP) { u0 += 0.5f * F0 * cp.dt; u1 += 0.5f * F1 * cp.dt; }
        else { const float h = cp.dt / (2.0f * rho); u0 += F0 * h; u1 += F1 * h; }
        collide32<COLL, INCOMP, true>(f, drho, rho, u0, u1, F0, F1, cp, out);
    } else {
        collide32<COLL, INCOMP, false>(f, drho, rho, u0, u1, 0.0f, 0.0f, cp, out);
    }
    if (OUT) {
        const long long n = (long long)j * g.nx + i;
        if (o.ro_out) o.ro_out[n] = rho;
        if (o.U_out) { o.U_out[2 * n] = u0; o.U_out[2 * n + 1] = u1; }
    }
    if (RING && is_ring(g, i, j)) {
        const long long n = (long long)j * g.nx + i;
        o.uring_next[2 * n] = u0;
        o.uring_next[2 * n + 1] = u1;
    }
}

// closures that extrapolate from the previous step's velocity ring
template <int BC>
__host__ __device__ constexpr bool has_ring() { return BC == BC_OPEN || BC == BC_VELOCITY_INLET; }

template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__device__ __forceinline__ void dense_node32(const float* __restrict__ fp, const float* __restrict__ ur, const Geom& g,
                                             const CollParams32& cp, const BcParams32& bc, const BandView32& band,
                                             const DenseOut32& o, int i, int j)
{
    float f[9], out[9];
    gstar_node<BC>(fp, ur, g, bc, INCOMP, i, j, f);
    node_core32<COLL, has_ring<BC>(), INCOMP, IBM, OUT>(f, g, cp, band, o, i, j, out);
    const long long site = (long long)j * g.pitch + i;
#pragma unroll
    for (int q = 0; q < 9; ++q) o.fpost_next[q * g.qstride + site] = out[q];
}

}  // namespace iblbm
