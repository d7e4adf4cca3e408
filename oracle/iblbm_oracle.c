/*
 * iblbm_oracle.c — CPU oracle for the IB-LBM per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the FP64 CPU path
 * of the reference solver (mulgae-life/iblbm-mechanism-resolved, numba + numpy
 * kernels selected by IBLBM_GPU=0).  It is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.  The product never links or calls it.
 *
 * Parity pin: tests/golden/ holds fixtures generated by running the reference
 * itself (tests/golden/make_golden.py); tests/test_oracle_golden.py checks this
 * oracle against them bit for bit.
 *
 * Arithmetic contract.  Every function evaluates the same expression trees, in
 * the same order, as the reference function it cites, with no FMA contraction
 * (built with -ffp-contract=off).  Reductions follow the reference's order:
 *   - numba loops accumulate sequentially over i = 0..8;
 *   - numpy `sum(axis=1)` over 9 entries is ((a0+a1)+(a2+a3))+((a4+a5)+(a6+a7)) + a8;
 *   - numpy `add.at` accumulates contributions in index order, i.e. stencil
 *     offset (di outer, dj inner) then marker l ascending.
 * Multiplications by the lattice vectors e_i in {0, +-1} are exact, so they are
 * written as the additions/subtractions they reduce to.
 *
 * Layout: the reference's own AoS layout, f[n*9 + q] with node n = j*nx + i
 * (iblbm/boundary/indices.py:3-5), U[n*2 + c].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

/* D2Q9: iblbm/lbm/lattice.py:45-55 — order 0; E,N,W,S; NE,NW,SW,SE */
static const int EX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int EY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int OPP[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const double W[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                            1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};

/* e_i . u with e in {0,+-1}: same value as e0*u0 + e1*u1 (products exact). */
static inline double e_dot(int q, double u0, double u1)
{
    double a = (double)EX[q] * u0;
    double b = (double)EY[q] * u1;
    return a + b;
}

/* ------------------------------------------------------------------------- */
/* Equilibrium — iblbm/lbm/equilibrium.py:27-43 (_compute_feq_nb)             */
/* ------------------------------------------------------------------------- */
static inline void feq_node(double ro, double u0, double u1, int incomp, double *out)
{
    double u2 = u0 * u0 + u1 * u1;
    for (int i = 0; i < 9; ++i) {
        double eU = e_dot(i, u0, u1);
        if (incomp)
            out[i] = W[i] * (ro + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
        else
            out[i] = ro * W[i] * (1.0 + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
    }
}

void orc_feq(int N, const double *ro, const double *U, int incomp, double *feq)
{
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n)
        feq_node(ro[n], U[2 * n], U[2 * n + 1], incomp, feq + 9 * (size_t)n);
}

/* ------------------------------------------------------------------------- */
/* Macroscopic — iblbm/lbm/macroscopic.py:27-49 (_macroscopic_nb)             */
/* sequential i = 0..8 accumulation                                          */
/* ------------------------------------------------------------------------- */
static inline void macro_node(const double *f, int incomp, double *ro, double *u0, double *u1)
{
    double s = 0.0, ux = 0.0, uy = 0.0;
    for (int i = 0; i < 9; ++i) {
        s += f[i];
        ux += f[i] * (double)EX[i];
        uy += f[i] * (double)EY[i];
    }
    *ro = s;
    if (incomp) {
        *u0 = ux;
        *u1 = uy;
    } else {
        *u0 = ux / s;
        *u1 = uy / s;
    }
}

void orc_macro(int N, const double *f, int incomp, double *ro, double *U)
{
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n)
        macro_node(f + 9 * (size_t)n, incomp, ro + n, U + 2 * n, U + 2 * n + 1);
}

/* ------------------------------------------------------------------------- */
/* BGK + Guo — iblbm/lbm/collision/bgk.py:25-40 (_collision_bgk_nb)           */
/* ------------------------------------------------------------------------- */
void orc_collide_bgk(int N, const double *fstar, const double *feq, const double *U,
                     const double *fib, double tau, double dt, double *f)
{
    const double inv_tau = 1.0 / tau;
    const double guo_pref = 1.0 - 0.5 / tau;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
        const double u0 = U[2 * n], u1 = U[2 * n + 1];
        const double F0 = fib[2 * n], F1 = fib[2 * n + 1];
        for (int i = 0; i < 9; ++i) {
            double ex = (double)EX[i], ey = (double)EY[i];
            double ax = ex - u0;
            double ay = ey - u1;
            double eU = ex * u0 + ey * u1;
            double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
            double F_ni = guo_pref * W[i] * term;
            size_t k = 9 * (size_t)n + i;
            f[k] = fstar[k] - inv_tau * (fstar[k] - feq[k]) + F_ni * dt;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* TRT + Guo — iblbm/lbm/collision/trt.py:38-67 (_collision_trt_nb)           */
/* s_plus = 1/tau, s_minus = 1/tau_minus (trt.py:80-86)                       */
/* ------------------------------------------------------------------------- */
void orc_collide_trt(int N, const double *fstar, const double *feq, const double *U,
                     const double *fib, double s_plus, double s_minus, double dt, double *f)
{
    const double gp = 1.0 - 0.5 * s_plus;
    const double gm = 1.0 - 0.5 * s_minus;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
        const double u0 = U[2 * n], u1 = U[2 * n + 1];
        const double F0 = fib[2 * n], F1 = fib[2 * n + 1];
        const double *fs = fstar + 9 * (size_t)n;
        const double *fe = feq + 9 * (size_t)n;
        double bare[9];
        for (int i = 0; i < 9; ++i) {
            double ex = (double)EX[i], ey = (double)EY[i];
            double ax = ex - u0;
            double ay = ey - u1;
            double eU = ex * u0 + ey * u1;
            double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
            bare[i] = W[i] * term;
        }
        for (int i = 0; i < 9; ++i) {
            int oi = OPP[i];
            double fp = 0.5 * (fs[i] + fs[oi]);
            double fm = 0.5 * (fs[i] - fs[oi]);
            double ep = 0.5 * (fe[i] + fe[oi]);
            double em = 0.5 * (fe[i] - fe[oi]);
            double coll = (s_plus * (fp - ep) + s_minus * (fm - em));
            double bp = 0.5 * (bare[i] + bare[oi]);
            double bm = 0.5 * (bare[i] - bare[oi]);
            double F_ni = gp * bp + gm * bm;
            f[9 * (size_t)n + i] = fs[i] - coll + F_ni * dt;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Central-moment MRT + Guo — iblbm/lbm/collision/cm_mrt.py:52-165            */
/* ------------------------------------------------------------------------- */
void orc_collide_cmmrt(int N, const double *fstar, const double *U, const double *fib,
                       const double *S, double dt, double *f_out)
{
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
        const double ux = U[2 * n], uy = U[2 * n + 1];
        const double F0 = fib[2 * n], F1 = fib[2 * n + 1];
        const double *fs = fstar + 9 * (size_t)n;
        double cm0 = 0.0, cm1 = 0.0, cm2 = 0.0, cm3 = 0.0, cm4 = 0.0, cm5 = 0.0, cm6 = 0.0,
               cm7 = 0.0, cm8 = 0.0;
        double Fc0 = 0.0, Fc1 = 0.0, Fc2 = 0.0, Fc3 = 0.0, Fc4 = 0.0, Fc5 = 0.0, Fc6 = 0.0,
               Fc7 = 0.0, Fc8 = 0.0;
        for (int i = 0; i < 9; ++i) {
            double val = fs[i];
            double ex = (double)EX[i], ey = (double)EY[i];
            double cix = ex - ux;
            double ciy = ey - uy;
            double cix2 = cix * cix;
            double ciy2 = ciy * ciy;
            cm0 += val;
            cm1 += val * cix;
            cm2 += val * ciy;
            cm3 += val * cix2;
            cm4 += val * ciy2;
            cm5 += val * cix * ciy;
            cm6 += val * cix2 * ciy;
            cm7 += val * cix * ciy2;
            cm8 += val * cix2 * ciy2;
            double ax = ex - ux;
            double ay = ey - uy;
            double eU = ex * ux + ey * uy;
            double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
            double Fb = W[i] * term;
            Fc0 += Fb;
            Fc1 += Fb * cix;
            Fc2 += Fb * ciy;
            Fc3 += Fb * cix2;
            Fc4 += Fb * ciy2;
            Fc5 += Fb * cix * ciy;
            Fc6 += Fb * cix2 * ciy;
            Fc7 += Fb * cix * ciy2;
            Fc8 += Fb * cix2 * ciy2;
        }
        const double rho = cm0;
        const double cs2 = 1.0 / 3.0;
        const double cs4 = 1.0 / 9.0;
        double cp0 = cm0 - S[0] * (cm0 - rho) + (1.0 - 0.5 * S[0]) * Fc0 * dt;
        double cp1 = cm1 - S[1] * (cm1 - 0.0) + (1.0 - 0.5 * S[1]) * Fc1 * dt;
        double cp2 = cm2 - S[2] * (cm2 - 0.0) + (1.0 - 0.5 * S[2]) * Fc2 * dt;
        double cp3 = cm3 - S[3] * (cm3 - rho * cs2) + (1.0 - 0.5 * S[3]) * Fc3 * dt;
        double cp4 = cm4 - S[4] * (cm4 - rho * cs2) + (1.0 - 0.5 * S[4]) * Fc4 * dt;
        double cp5 = cm5 - S[5] * (cm5 - 0.0) + (1.0 - 0.5 * S[5]) * Fc5 * dt;
        double cp6 = cm6 - S[6] * (cm6 - 0.0) + (1.0 - 0.5 * S[6]) * Fc6 * dt;
        double cp7 = cm7 - S[7] * (cm7 - 0.0) + (1.0 - 0.5 * S[7]) * Fc7 * dt;
        double cp8 = cm8 - S[8] * (cm8 - rho * cs4) + (1.0 - 0.5 * S[8]) * Fc8 * dt;
        double ux2 = ux * ux;
        double uy2 = uy * uy;
        double k0 = cp0;
        double k1 = cp1 + ux * cp0;
        double k2 = cp2 + uy * cp0;
        double k3 = cp3 + 2.0 * ux * cp1 + ux2 * cp0;
        double k4 = cp4 + 2.0 * uy * cp2 + uy2 * cp0;
        double k5 = cp5 + uy * cp1 + ux * cp2 + ux * uy * cp0;
        double k6 = (cp6 + uy * cp3 + 2.0 * ux * cp5 + 2.0 * ux * uy * cp1 + ux2 * cp2 + ux2 * uy * cp0);
        double k7 = (cp7 + 2.0 * uy * cp5 + ux * cp4 + 2.0 * ux * uy * cp2 + uy2 * cp1 + ux * uy2 * cp0);
        double k8 = (cp8 + 2.0 * uy * cp6 + uy2 * cp3 + 2.0 * ux * cp7 + 4.0 * ux * uy * cp5 +
                     2.0 * ux * uy2 * cp1 + ux2 * cp4 + 2.0 * ux2 * uy * cp2 + ux2 * uy2 * cp0);
        double *fo = f_out + 9 * (size_t)n;
        fo[0] = k0 - k3 - k4 + k8;
        fo[1] = 0.5 * (k1 + k3 - k7 - k8);
        fo[2] = 0.5 * (k2 + k4 - k6 - k8);
        fo[3] = 0.5 * (-k1 + k3 + k7 - k8);
        fo[4] = 0.5 * (-k2 + k4 + k6 - k8);
        fo[5] = 0.25 * (k5 + k6 + k7 + k8);
        fo[6] = 0.25 * (-k5 + k6 - k7 + k8);
        fo[7] = 0.25 * (k5 - k6 - k7 + k8);
        fo[8] = 0.25 * (-k5 - k6 + k7 + k8);
    }
}

/* ------------------------------------------------------------------------- */
/* Streaming — iblbm/lbm/streaming.py:38-77 (_streaming_step_nb)             */
/* push form; a population whose source lies outside the lattice keeps its   */
/* previous post-streaming value (fstar_new starts as a copy of fstar_old)   */
/* ------------------------------------------------------------------------- */
void orc_stream(int nx, int ny, const double *fstar_old, const double *f, double *fstar_new)
{
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
            size_t n = (size_t)j * nx + i;
            for (int q = 0; q < 9; ++q) {
                int si = i - EX[q], sj = j - EY[q];
                if (si < 0 || si >= nx || sj < 0 || sj >= ny)
                    fstar_new[9 * n + q] = fstar_old[9 * n + q];
                else
                    fstar_new[9 * n + q] = f[9 * ((size_t)sj * nx + si) + q];
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Boundary closures                                                         */
/* ------------------------------------------------------------------------- */
#define FS(n, q) fstar[9 * (size_t)(n) + (q)]
#define UX(n) U[2 * (size_t)(n)]
#define UY(n) U[2 * (size_t)(n) + 1]

/* numpy row sum over 9 entries (pairwise order), used by dirichlet_neumann */
static inline double np_sum9(const double *a)
{
    double r = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    return r + a[8];
}

/* _macro_from_streamed — iblbm/boundary/dirichlet_neumann.py:63-69 */
static inline void dn_macro(const double *f, double *ro, double *u0, double *u1)
{
    double px[9], py[9];
    for (int i = 0; i < 9; ++i) {
        px[i] = f[i] * (double)EX[i];
        py[i] = f[i] * (double)EY[i];
    }
    double r = np_sum9(f);
    *ro = r;
    *u0 = np_sum9(px) / r;
    *u1 = np_sum9(py) / r;
}

/* iblbm/boundary/dirichlet_neumann.py:39-120 */
void orc_bc_dirichlet_neumann(int nx, int ny, double *fstar, double *ro, double *U,
                              double inflow_u, double dens)
{
    double fe[9];
    /* left (corners excluded), top, bottom: f <- feq(dens, (u_in, 0)) */
    feq_node(dens, inflow_u, 0.0, 0, fe);
    for (int j = 1; j <= ny - 2; ++j) {
        size_t n = (size_t)j * nx;
        ro[n] = dens; UX(n) = inflow_u; UY(n) = 0.0;
        memcpy(&FS(n, 0), fe, sizeof fe);
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)(ny - 1) * nx + i;
        ro[n] = dens; UX(n) = inflow_u; UY(n) = 0.0;
        memcpy(&FS(n, 0), fe, sizeof fe);
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)i;
        ro[n] = dens; UX(n) = inflow_u; UY(n) = 0.0;
        memcpy(&FS(n, 0), fe, sizeof fe);
    }
    /* right (Neumann): copy non-equilibrium part from right_inner = right - 1 */
    for (int j = 1; j <= ny - 2; ++j) {
        size_t n = (size_t)j * nx + nx - 1, m = n - 1;
        double r, a, b, fq[9];
        dn_macro(&FS(m, 0), &r, &a, &b);
        ro[n] = r; UX(n) = a; UY(n) = b;
        feq_node(r, a, b, 0, fq);
        for (int q = 0; q < 9; ++q) FS(n, q) = fq[q] + (FS(m, q) - fq[q]);
    }
    /* left corners: Dirichlet refill */
    size_t lc[2] = {0, (size_t)nx * (ny - 1)};
    for (int c = 0; c < 2; ++c) {
        ro[lc[c]] = dens; UX(lc[c]) = inflow_u; UY(lc[c]) = 0.0;
        memcpy(&FS(lc[c], 0), fe, sizeof fe);
    }
    /* right corners: Neumann copy from the diagonal interior nodes */
    size_t rc[2] = {(size_t)nx - 1, (size_t)nx * ny - 1};
    size_t rd[2] = {2 * (size_t)nx - 2, (size_t)nx * (ny - 1) - 2};
    double rr[2], ra[2], rb[2];
    for (int c = 0; c < 2; ++c) dn_macro(&FS(rd[c], 0), &rr[c], &ra[c], &rb[c]);
    for (int c = 0; c < 2; ++c) {
        double fq[9];
        ro[rc[c]] = rr[c]; UX(rc[c]) = ra[c]; UY(rc[c]) = rb[c];
        feq_node(rr[c], ra[c], rb[c], 0, fq);
        for (int q = 0; q < 9; ++q) FS(rc[c], q) = fq[q] + (FS(rd[c], q) - fq[q]);
    }
}

/* iblbm/boundary/open_boundary.py:44-165 — pressure on all four faces.
 * The tangential extrapolations read U from the previous step (U on entry). */
void orc_bc_open_boundary(int nx, int ny, double *fstar, double *ro, double *U, double dens)
{
    /* left: i = 0, j in [1, ny-2] */
    for (int j = 1; j <= ny - 2; ++j) {
        size_t n = (size_t)j * nx;
        ro[n] = dens;
        UX(n) = 1.0 - (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 3) + FS(n, 7) + FS(n, 6))) / ro[n];
        UY(n) = (4.0 * UY(n + 1) - UY(n + 2)) / 3.0;
        FS(n, 1) = FS(n, 3) + (2.0 / 3.0) * ro[n] * UX(n);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 2) - FS(n, 4)) + (1.0 / 6.0) * ro[n] * UX(n) + 0.5 * ro[n] * UY(n));
        FS(n, 8) = (FS(n, 6) + 0.5 * (FS(n, 2) - FS(n, 4)) + (1.0 / 6.0) * ro[n] * UX(n) - 0.5 * ro[n] * UY(n));
    }
    /* right: i = nx-1 */
    for (int j = 1; j <= ny - 2; ++j) {
        size_t n = (size_t)j * nx + nx - 1;
        ro[n] = dens;
        UX(n) = -1.0 + (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 1) + FS(n, 5) + FS(n, 8))) / ro[n];
        UY(n) = (4.0 * UY(n - 1) - UY(n - 2)) / 3.0;
        FS(n, 3) = FS(n, 1) - (2.0 / 3.0) * ro[n] * UX(n);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 2) - FS(n, 4)) - (1.0 / 6.0) * ro[n] * UX(n) - 0.5 * ro[n] * UY(n));
        FS(n, 6) = (FS(n, 8) - 0.5 * (FS(n, 2) - FS(n, 4)) - (1.0 / 6.0) * ro[n] * UX(n) + 0.5 * ro[n] * UY(n));
    }
    /* top: j = ny-1, i in [1, nx-2] */
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)(ny - 1) * nx + i;
        ro[n] = dens;
        UY(n) = -1.0 + (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 2) + FS(n, 5) + FS(n, 6))) / ro[n];
        UX(n) = (4.0 * UX(n - nx) - UX(n - 2 * (size_t)nx)) / 3.0;
        FS(n, 4) = FS(n, 2) - (2.0 / 3.0) * ro[n] * UY(n);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 1) - FS(n, 3)) - (1.0 / 6.0) * ro[n] * UY(n) - 0.5 * ro[n] * UX(n));
        FS(n, 8) = (FS(n, 6) - 0.5 * (FS(n, 1) - FS(n, 3)) - (1.0 / 6.0) * ro[n] * UY(n) + 0.5 * ro[n] * UX(n));
    }
    /* bottom: j = 0 */
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)i;
        ro[n] = dens;
        UY(n) = 1.0 - (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 4) + FS(n, 7) + FS(n, 8))) / ro[n];
        UX(n) = (4.0 * UX(n + nx) - UX(n + 2 * (size_t)nx)) / 3.0;
        FS(n, 2) = FS(n, 4) + (2.0 / 3.0) * ro[n] * UY(n);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 1) - FS(n, 3)) + (1.0 / 6.0) * ro[n] * UY(n) + 0.5 * ro[n] * UX(n));
        FS(n, 6) = (FS(n, 8) + 0.5 * (FS(n, 1) - FS(n, 3)) + (1.0 / 6.0) * ro[n] * UY(n) - 0.5 * ro[n] * UX(n));
    }
    /* corners: U copied from the diagonal interior nodes, equilibrium refill */
    size_t corners[4] = {0, (size_t)nx - 1, (size_t)nx * (ny - 1), (size_t)nx * ny - 1};
    size_t diag1[4] = {(size_t)nx + 1, 2 * (size_t)nx - 2, (size_t)nx * (ny - 2) + 1,
                       (size_t)nx * (ny - 1) - 2};
    double cu[4][2];
    for (int c = 0; c < 4; ++c) { cu[c][0] = UX(diag1[c]); cu[c][1] = UY(diag1[c]); }
    for (int c = 0; c < 4; ++c) {
        ro[corners[c]] = dens;
        UX(corners[c]) = cu[c][0];
        UY(corners[c]) = cu[c][1];
        feq_node(dens, cu[c][0], cu[c][1], 0, &FS(corners[c], 0));
    }
}

/* iblbm/boundary/settling_channel.py:42-145 — no-slip on all four walls */
void orc_bc_settling_channel(int nx, int ny, double *fstar, double *ro, double *U, double dens,
                             int incomp)
{
    for (int j = 1; j <= ny - 2; ++j) {
        size_t n = (size_t)j * nx;
        UX(n) = 0.0; UY(n) = 0.0;
        ro[n] = (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 3) + FS(n, 6) + FS(n, 7)));
        FS(n, 1) = FS(n, 3);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 2) - FS(n, 4)));
        FS(n, 8) = (FS(n, 6) + 0.5 * (FS(n, 2) - FS(n, 4)));
    }
    for (int j = 1; j <= ny - 2; ++j) {
        size_t n = (size_t)j * nx + nx - 1;
        UX(n) = 0.0; UY(n) = 0.0;
        ro[n] = (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 1) + FS(n, 5) + FS(n, 8)));
        FS(n, 3) = FS(n, 1);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 2) - FS(n, 4)));
        FS(n, 6) = (FS(n, 8) - 0.5 * (FS(n, 2) - FS(n, 4)));
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)(ny - 1) * nx + i;
        UX(n) = 0.0; UY(n) = 0.0;
        ro[n] = (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 2) + FS(n, 5) + FS(n, 6)));
        FS(n, 4) = FS(n, 2);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 1) - FS(n, 3)));
        FS(n, 8) = (FS(n, 6) - 0.5 * (FS(n, 1) - FS(n, 3)));
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)i;
        UX(n) = 0.0; UY(n) = 0.0;
        ro[n] = (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 4) + FS(n, 7) + FS(n, 8)));
        FS(n, 2) = FS(n, 4);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 1) - FS(n, 3)));
        FS(n, 6) = (FS(n, 8) + 0.5 * (FS(n, 1) - FS(n, 3)));
    }
    size_t corners[4] = {0, (size_t)nx - 1, (size_t)nx * (ny - 1), (size_t)nx * ny - 1};
    for (int c = 0; c < 4; ++c) {
        ro[corners[c]] = dens; UX(corners[c]) = 0.0; UY(corners[c]) = 0.0;
        feq_node(dens, 0.0, 0.0, incomp, &FS(corners[c], 0));
    }
}

/* iblbm/boundary/velocity_inlet.py:45-160 — left/right faces include the corners */
void orc_bc_velocity_inlet(int nx, int ny, double *fstar, double *ro, double *U, double inflow_u,
                           double dens)
{
    for (int j = 0; j <= ny - 1; ++j) {
        size_t n = (size_t)j * nx;
        UX(n) = inflow_u; UY(n) = 0.0;
        ro[n] = (1.0 / (1.0 - UX(n))) * (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 3) + FS(n, 6) + FS(n, 7)));
        FS(n, 1) = FS(n, 3) + (2.0 / 3.0) * ro[n] * UX(n);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 2) - FS(n, 4)) + (1.0 / 6.0) * ro[n] * UX(n) + 0.5 * ro[n] * UY(n));
        FS(n, 8) = (FS(n, 6) + 0.5 * (FS(n, 2) - FS(n, 4)) + (1.0 / 6.0) * ro[n] * UX(n) - 0.5 * ro[n] * UY(n));
    }
    /* right: ro = dens, U_y extrapolated from the previous step's U */
    double *uyr = (double *)malloc(sizeof(double) * (size_t)ny);
    for (int j = 0; j <= ny - 1; ++j) {
        size_t n = (size_t)j * nx + nx - 1;
        uyr[j] = (4.0 * UY(n - 1) - UY(n - 2)) / 3.0;
    }
    for (int j = 0; j <= ny - 1; ++j) {
        size_t n = (size_t)j * nx + nx - 1;
        ro[n] = dens;
        UX(n) = -1.0 + (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 1) + FS(n, 5) + FS(n, 8))) / ro[n];
        UY(n) = uyr[j];
        FS(n, 3) = FS(n, 1) - (2.0 / 3.0) * ro[n] * UX(n);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 2) - FS(n, 4)) - (1.0 / 6.0) * ro[n] * UX(n) - 0.5 * ro[n] * UY(n));
        FS(n, 6) = (FS(n, 8) - 0.5 * (FS(n, 2) - FS(n, 4)) - (1.0 / 6.0) * ro[n] * UX(n) + 0.5 * ro[n] * UY(n));
    }
    free(uyr);
    double *uxt = (double *)malloc(sizeof(double) * (size_t)nx);
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)(ny - 1) * nx + i;
        uxt[i] = (4.0 * UX(n - nx) - UX(n - 2 * (size_t)nx)) / 3.0;
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)(ny - 1) * nx + i;
        UX(n) = uxt[i]; UY(n) = 0.0;
        ro[n] = (1.0 / (1.0 + UY(n))) * (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 2) + FS(n, 5) + FS(n, 6)));
        FS(n, 4) = FS(n, 2) - (2.0 / 3.0) * ro[n] * UY(n);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 1) - FS(n, 3)) - 0.5 * ro[n] * UX(n));
        FS(n, 8) = (FS(n, 6) - 0.5 * (FS(n, 1) - FS(n, 3)) + 0.5 * ro[n] * UX(n));
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)i;
        uxt[i] = (4.0 * UX(n + nx) - UX(n + 2 * (size_t)nx)) / 3.0;
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)i;
        UX(n) = uxt[i]; UY(n) = 0.0;
        ro[n] = (1.0 / (1.0 - UY(n))) * (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 4) + FS(n, 7) + FS(n, 8)));
        FS(n, 2) = FS(n, 4) + (2.0 / 3.0) * ro[n] * UY(n);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 1) - FS(n, 3)) + 0.5 * ro[n] * UX(n));
        FS(n, 6) = (FS(n, 8) + 0.5 * (FS(n, 1) - FS(n, 3)) - 0.5 * ro[n] * UX(n));
    }
    free(uxt);
    /* inlet corners */
    size_t ic[2] = {0, (size_t)(ny - 1) * nx};
    for (int c = 0; c < 2; ++c) {
        ro[ic[c]] = dens; UX(ic[c]) = inflow_u; UY(ic[c]) = 0.0;
        feq_node(dens, inflow_u, 0.0, 0, &FS(ic[c], 0));
    }
    /* outlet corners: sequential loop over ci (velocity_inlet.py:153-155) */
    size_t oc[2] = {(size_t)nx - 1, (size_t)(ny - 1) * nx + nx - 1};
    for (int c = 0; c < 2; ++c) ro[oc[c]] = dens;
    for (int c = 0; c < 2; ++c) UX(oc[c]) = (4.0 * UX(oc[c] - 1) - UX(oc[c] - 2)) / 3.0;
    for (int c = 0; c < 2; ++c) UY(oc[c]) = 0.0;
    for (int c = 0; c < 2; ++c) feq_node(dens, UX(oc[c]), 0.0, 0, &FS(oc[c], 0));
}

/* iblbm/boundary/tg_analytical.py:26-170 — time-dependent Dirichlet on all four faces
 * (Zou-He closures with the analytic velocity), then the four corners reset to
 * feq(1, u).  The analytic velocities at this step come in per face: uL, uR over
 * j = 0..ny-1 (the faces include the corners), uB, uT over i = 1..nx-2, uC for
 * the corners (0,0), (nx-1,0), (0,ny-1), (nx-1,ny-1); each as (ux, uy) pairs. */
void orc_bc_tg(int nx, int ny, double *fstar, double *ro, double *U, const double *uL, const double *uR,
               const double *uB, const double *uT, const double *uC)
{
    for (int j = 0; j <= ny - 1; ++j) {
        size_t n = (size_t)j * nx;
        UX(n) = uL[2 * j]; UY(n) = uL[2 * j + 1];
        ro[n] = (1.0 / (1.0 - UX(n))) * (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 3) + FS(n, 6) + FS(n, 7)));
        FS(n, 1) = FS(n, 3) + (2.0 / 3.0) * ro[n] * UX(n);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 2) - FS(n, 4)) + (1.0 / 6.0) * ro[n] * UX(n) + 0.5 * ro[n] * UY(n));
        FS(n, 8) = (FS(n, 6) + 0.5 * (FS(n, 2) - FS(n, 4)) + (1.0 / 6.0) * ro[n] * UX(n) - 0.5 * ro[n] * UY(n));
    }
    for (int j = 0; j <= ny - 1; ++j) {
        size_t n = (size_t)j * nx + nx - 1;
        UX(n) = uR[2 * j]; UY(n) = uR[2 * j + 1];
        ro[n] = (1.0 / (1.0 + UX(n))) * (FS(n, 0) + FS(n, 2) + FS(n, 4) + 2.0 * (FS(n, 1) + FS(n, 5) + FS(n, 8)));
        FS(n, 3) = FS(n, 1) - (2.0 / 3.0) * ro[n] * UX(n);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 2) - FS(n, 4)) - (1.0 / 6.0) * ro[n] * UX(n) - 0.5 * ro[n] * UY(n));
        FS(n, 6) = (FS(n, 8) - 0.5 * (FS(n, 2) - FS(n, 4)) - (1.0 / 6.0) * ro[n] * UX(n) + 0.5 * ro[n] * UY(n));
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)(ny - 1) * nx + i;
        UX(n) = uT[2 * (i - 1)]; UY(n) = uT[2 * (i - 1) + 1];
        ro[n] = (1.0 / (1.0 + UY(n))) * (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 2) + FS(n, 5) + FS(n, 6)));
        FS(n, 4) = FS(n, 2) - (2.0 / 3.0) * ro[n] * UY(n);
        FS(n, 7) = (FS(n, 5) + 0.5 * (FS(n, 1) - FS(n, 3)) - (1.0 / 6.0) * ro[n] * UY(n) - 0.5 * ro[n] * UX(n));
        FS(n, 8) = (FS(n, 6) - 0.5 * (FS(n, 1) - FS(n, 3)) - (1.0 / 6.0) * ro[n] * UY(n) + 0.5 * ro[n] * UX(n));
    }
    for (int i = 1; i <= nx - 2; ++i) {
        size_t n = (size_t)i;
        UX(n) = uB[2 * (i - 1)]; UY(n) = uB[2 * (i - 1) + 1];
        ro[n] = (1.0 / (1.0 - UY(n))) * (FS(n, 0) + FS(n, 1) + FS(n, 3) + 2.0 * (FS(n, 4) + FS(n, 7) + FS(n, 8)));
        FS(n, 2) = FS(n, 4) + (2.0 / 3.0) * ro[n] * UY(n);
        FS(n, 5) = (FS(n, 7) - 0.5 * (FS(n, 1) - FS(n, 3)) + (1.0 / 6.0) * ro[n] * UY(n) + 0.5 * ro[n] * UX(n));
        FS(n, 6) = (FS(n, 8) + 0.5 * (FS(n, 1) - FS(n, 3)) + (1.0 / 6.0) * ro[n] * UY(n) - 0.5 * ro[n] * UX(n));
    }
    size_t corners[4] = {0, (size_t)nx - 1, (size_t)nx * (ny - 1), (size_t)nx * ny - 1};
    for (int c = 0; c < 4; ++c) {
        size_t n = corners[c];
        ro[n] = 1.0; UX(n) = uC[2 * c]; UY(n) = uC[2 * c + 1];
        feq_node(1.0, UX(n), UY(n), 0, &FS(n, 0));
    }
}

/* bc_type ids: 0 dirichlet_neumann, 1 open_boundary, 2 settling_channel, 3 velocity_inlet */
int orc_bc(int bc_type, int nx, int ny, double *fstar, double *ro, double *U, double inflow_u,
           double dens, int incomp)
{
    switch (bc_type) {
    case 0: orc_bc_dirichlet_neumann(nx, ny, fstar, ro, U, inflow_u, dens); return 0;
    case 1: orc_bc_open_boundary(nx, ny, fstar, ro, U, dens); return 0;
    case 2: orc_bc_settling_channel(nx, ny, fstar, ro, U, dens, incomp); return 0;
    case 3: orc_bc_velocity_inlet(nx, ny, fstar, ro, U, inflow_u, dens); return 0;
    default: return -1;
    }
}

/* ------------------------------------------------------------------------- */
/* Velocity correction — iblbm/ibm/dispatch.py:18-33 (CPU branch)             */
/* ------------------------------------------------------------------------- */
void orc_velocity_correction(int N, double *U, const double *fib, const double *ro, double dt,
                             int incomp)
{
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
        for (int c = 0; c < 2; ++c) {
            if (incomp)
                U[2 * n + c] = U[2 * n + c] + 0.5 * fib[2 * n + c] * dt;
            else
                U[2 * n + c] = U[2 * n + c] + fib[2 * n + c] * dt / (2.0 * ro[n]);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Delta kernels — iblbm/ibm/common.py:52-119                                */
/* ------------------------------------------------------------------------- */
static inline double phi_hat(double r)
{
    double v = 1.0 - fabs(r);
    return v > 0.0 ? v : 0.0; /* np.maximum(., 0.0) */
}

static inline double phi_p4(double r)
{
    double ar = fabs(r);
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

/* delta_type ids: 0 peskin4pt (a = 2), 1 hat (a = 1) — gpu_kernels.py:952-953 naming */
static inline double phi(int delta_type, double r)
{
    return delta_type == 0 ? phi_p4(r) : phi_hat(r);
}

static inline int stencil_a(int delta_type) { return delta_type == 0 ? 2 : 1; }

static inline long clipl(long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Stencil of one marker: ix0 = floor(Lx/dx + 0.5); weights per (di, dj) in
 * (di outer, dj inner) order; clipped node index.  iblbm/ibm/df.py:94-118. */
typedef struct {
    int count;
    long node[25];
    double w[25]; /* wx * wy (without Larea) */
} stencil_t;

static void marker_stencil(double Lx, double Ly, double dx, double dy, int nx, int ny,
                           int delta_type, stencil_t *st)
{
    int a = stencil_a(delta_type);
    long ix0 = (long)floor(Lx / dx + 0.5);
    long iy0 = (long)floor(Ly / dy + 0.5);
    int k = 0;
    for (int di = -a; di <= a; ++di) {
        for (int dj = -a; dj <= a; ++dj) {
            long ei = ix0 + di, ej = iy0 + dj;
            long eic = clipl(ei, 0, nx - 1), ejc = clipl(ej, 0, ny - 1);
            double wx = phi(delta_type, (Lx - (double)ei * dx) / dx);
            double wy = phi(delta_type, (Ly - (double)ej * dy) / dy);
            st->node[k] = ejc * nx + eic;
            st->w[k] = wx * wy;
            ++k;
        }
    }
    st->count = k;
}

/* ------------------------------------------------------------------------- */
/* Direct forcing — iblbm/ibm/df.py:37-154 (CPU branch, lines 93-154)         */
/* Outputs fib (N x 2, dense, zero outside the stencils) and per marker       */
/* Lux, Luy, Lfx, Lfy, R.                                                     */
/* ------------------------------------------------------------------------- */
void orc_ibm_df(int nx, int ny, int Lb, const double *Lx, const double *Ly,
                const double *dvel, const double *Eux, const double *Euy, const double *Ro,
                double dx, double dy, double dt, double Larea, int delta_type, int incomp,
                double *fib, double *Lux, double *Luy, double *Lfx, double *Lfy, double *R)
{
    size_t N = (size_t)nx * ny;
    stencil_t *st = (stencil_t *)malloc(sizeof(stencil_t) * (size_t)(Lb > 0 ? Lb : 1));
    for (int l = 0; l < Lb; ++l) marker_stencil(Lx[l], Ly[l], dx, dy, nx, ny, delta_type, &st[l]);
    int S = Lb > 0 ? st[0].count : 0;
    for (int l = 0; l < Lb; ++l) { R[l] = 0.0; Lux[l] = 0.0; Luy[l] = 0.0; }
    for (int k = 0; k < S; ++k) {
        for (int l = 0; l < Lb; ++l) {
            long n = st[l].node[k];
            double w = st[l].w[k];
            R[l] += Ro[n] * w;
            Lux[l] += Eux[n] * w;
            Luy[l] += Euy[n] * w;
        }
    }
    for (int l = 0; l < Lb; ++l) {
        if (incomp) {
            Lfx[l] = 2.0 * (dvel[2 * l] - Lux[l]) / dt;
            Lfy[l] = 2.0 * (dvel[2 * l + 1] - Luy[l]) / dt;
        } else {
            Lfx[l] = 2.0 * R[l] * (dvel[2 * l] - Lux[l]) / dt;
            Lfy[l] = 2.0 * R[l] * (dvel[2 * l + 1] - Luy[l]) / dt;
        }
    }
    memset(fib, 0, sizeof(double) * 2 * N);
    for (int k = 0; k < S; ++k) {
        for (int l = 0; l < Lb; ++l) {
            long n = st[l].node[k];
            double w = st[l].w[k] * Larea;
            fib[2 * n] += Lfx[l] * w;
            fib[2 * n + 1] += Lfy[l] * w;
        }
    }
    free(st);
}

/* ------------------------------------------------------------------------- */
/* Multi-direct forcing — iblbm/ibm/mdf.py:61-229 (CPU branch, lines 170-229)  */
/* U is AoS (N x 2); ro (N).  The force law is always the compressible one    */
/* (mdf.py calls ibm_direct_forcing without `incompressible`).                */
/* stats: [iter_count, diverged, converged]; last_residual in *res_out.       */
/* ------------------------------------------------------------------------- */
void orc_ibm_mdf(int nx, int ny, int Lb, const double *Lx, const double *Ly, const double *dvel,
                 const double *U, const double *ro, double dx, double dy, double dt, double Larea,
                 int n_iter, int min_iter, int delta_type, double omega, double tol,
                 double *fib_total, int *stats, double *res_out)
{
    size_t N = (size_t)nx * ny;
    double *Eux = (double *)malloc(sizeof(double) * N);
    double *Euy = (double *)malloc(sizeof(double) * N);
    double *vs = (double *)malloc(sizeof(double) * N);
    double *fib = (double *)malloc(sizeof(double) * 2 * N);
    double *Lux = (double *)malloc(sizeof(double) * (size_t)Lb);
    double *Luy = (double *)malloc(sizeof(double) * (size_t)Lb);
    double *Lfx = (double *)malloc(sizeof(double) * (size_t)Lb);
    double *Lfy = (double *)malloc(sizeof(double) * (size_t)Lb);
    double *R = (double *)malloc(sizeof(double) * (size_t)Lb);
    for (size_t n = 0; n < N; ++n) {
        Eux[n] = U[2 * n];
        Euy[n] = U[2 * n + 1];
        vs[n] = dt / (2.0 * ro[n]);
    }
    if (min_iter > n_iter) min_iter = n_iter;
    if (min_iter < 1) min_iter = 1;
    double prev = INFINITY, last = INFINITY;
    int iter_count = 0, diverged = 0, converged = 0;
    memset(fib_total, 0, sizeof(double) * 2 * N);
    for (int it = 0; it < n_iter; ++it) {
        orc_ibm_df(nx, ny, Lb, Lx, Ly, dvel, Eux, Euy, ro, dx, dy, dt, Larea, delta_type, 0, fib,
                   Lux, Luy, Lfx, Lfy, R);
        double residual = -INFINITY;
        for (int l = 0; l < Lb; ++l) {
            double vx = dvel[2 * l] - Lux[l];
            double vy = dvel[2 * l + 1] - Luy[l];
            double r = sqrt(vx * vx + vy * vy);
            if (r > residual || r != r) residual = r;
        }
        last = residual;
        if (it > 0 && residual > prev * 1.5) {
            diverged = 1;
            iter_count = it + 1;
            break;
        }
        for (size_t n = 0; n < N; ++n) {
            double fx = fib[2 * n] * omega, fy = fib[2 * n + 1] * omega;
            fib_total[2 * n] += fx;
            fib_total[2 * n + 1] += fy;
            Eux[n] += fx * vs[n];
            Euy[n] += fy * vs[n];
        }
        prev = residual;
        iter_count = it + 1;
        if ((it + 1) >= min_iter && residual < tol) {
            converged = 1;
            break;
        }
    }
    stats[0] = iter_count;
    stats[1] = diverged;
    stats[2] = converged;
    *res_out = last;
    free(Eux); free(Euy); free(vs); free(fib); free(Lux); free(Luy); free(Lfx); free(Lfy); free(R);
}

/* ------------------------------------------------------------------------- */
/* Coupled multi-particle MDF — iblbm/ibm/multi_particle.py:62-316 (CPU branch */
/* lines 243-316).  Particles p = 0..P-1 own markers [moff[p], moff[p+1]).     */
/* Outputs fib_total (N x 2), per-particle force sums pforce (P x 2) equal to  */
/* -sum(fib_p) with the same dense-sum order as the reference (pairwise over  */
/* the strided column; computed by the caller), and stats.                    */
/* Here per-particle dense fib_p (P x N x 2) is returned so the caller can    */
/* form the reference's numpy sums.                                           */
/* stats: [iter_count, diverged, converged, guard_trips]; dstats: [last_res, omega_used] */
/* ------------------------------------------------------------------------- */
void orc_mdf_coupled(int nx, int ny, int P, const int *moff, const double *Lx, const double *Ly,
                     const double *dvel, const double *Larea, const double *U, const double *ro,
                     double dx, double dy, double dt, int n_iter, int min_iter_cfg,
                     int delta_type, double omega_opt, double omega_max, double tol, int incomp,
                     double *fib_total, double *fib_part, int *stats, double *dstats)
{
    size_t N = (size_t)nx * ny;
    int Lmax = 0;
    for (int p = 0; p < P; ++p) if (moff[p + 1] - moff[p] > Lmax) Lmax = moff[p + 1] - moff[p];
    double *Eux = (double *)malloc(sizeof(double) * N);
    double *Euy = (double *)malloc(sizeof(double) * N);
    double *vs = (double *)malloc(sizeof(double) * N);
    double *this_it = (double *)malloc(sizeof(double) * 2 * N);
    double *fp = (double *)malloc(sizeof(double) * 2 * N * (size_t)P);
    double *Lux = (double *)malloc(sizeof(double) * (size_t)Lmax);
    double *Luy = (double *)malloc(sizeof(double) * (size_t)Lmax);
    double *Lfx = (double *)malloc(sizeof(double) * (size_t)Lmax);
    double *Lfy = (double *)malloc(sizeof(double) * (size_t)Lmax);
    double *R = (double *)malloc(sizeof(double) * (size_t)Lmax);
    for (size_t n = 0; n < N; ++n) {
        Eux[n] = U[2 * n];
        Euy[n] = U[2 * n + 1];
        vs[n] = dt / (2.0 * ro[n]);
    }
    double omega_use = omega_opt * 0.8;
    if (omega_use > omega_max) omega_use = omega_max; /* min(omega_opt*0.8, MAX) */
    double omega_min = omega_use * 0.125;
    int guard = 0, iter_count = 0, diverged = 0, converged = 0;
    double last = INFINITY, prev = INFINITY;
    int min_iter = min_iter_cfg < n_iter ? min_iter_cfg : n_iter;
    if (min_iter < 1) min_iter = 1;
    memset(fib_total, 0, sizeof(double) * 2 * N);
    memset(fib_part, 0, sizeof(double) * 2 * N * (size_t)P);
    for (int it = 0; it < n_iter; ++it) {
        memset(this_it, 0, sizeof(double) * 2 * N);
        double residual_max = 0.0;
        for (int p = 0; p < P; ++p) {
            int Lb = moff[p + 1] - moff[p];
            int o = moff[p];
            double *fpp = fp + 2 * N * (size_t)p;
            orc_ibm_df(nx, ny, Lb, Lx + o, Ly + o, dvel + 2 * o, Eux, Euy, ro, dx, dy, dt,
                       Larea[p], delta_type, incomp, fpp, Lux, Luy, Lfx, Lfy, R);
            double res_p = -INFINITY;
            for (int l = 0; l < Lb; ++l) {
                double vx = dvel[2 * (o + l)] - Lux[l];
                double vy = dvel[2 * (o + l) + 1] - Luy[l];
                double r = sqrt(vx * vx + vy * vy);
                if (r > res_p || r != r) res_p = r;
            }
            /* residual_max = max(residual_max, float(res_p)) — Python builtin max */
            if (res_p > residual_max) residual_max = res_p;
            for (size_t k = 0; k < 2 * N; ++k) {
                fpp[k] *= omega_use;
                this_it[k] += fpp[k];
            }
        }
        if (it > 0 && residual_max > prev * 1.2) {
            guard += 1;
            double h = omega_use * 0.5;
            omega_use = h > omega_min ? h : omega_min;
            if (omega_use <= omega_min) {
                diverged = 1;
                break;
            }
            prev = residual_max;
            continue;
        }
        for (size_t k = 0; k < 2 * N; ++k) fib_total[k] += this_it[k];
        for (int p = 0; p < P; ++p) {
            double *acc = fib_part + 2 * N * (size_t)p;
            const double *src = fp + 2 * N * (size_t)p;
            for (size_t k = 0; k < 2 * N; ++k) acc[k] += src[k];
        }
        for (size_t n = 0; n < N; ++n) {
            if (incomp) {
                Eux[n] += 0.5 * this_it[2 * n] * dt;
                Euy[n] += 0.5 * this_it[2 * n + 1] * dt;
            } else {
                Eux[n] += this_it[2 * n] * vs[n];
                Euy[n] += this_it[2 * n + 1] * vs[n];
            }
        }
        prev = residual_max;
        iter_count += 1;
        last = residual_max;
        if ((it + 1) >= min_iter && residual_max < tol) {
            converged = 1;
            break;
        }
    }
    stats[0] = iter_count;
    stats[1] = diverged;
    stats[2] = converged;
    stats[3] = guard;
    dstats[0] = last;
    dstats[1] = omega_use;
    free(Eux); free(Euy); free(vs); free(this_it); free(fp);
    free(Lux); free(Luy); free(Lfx); free(Lfy); free(R);
}

/* ------------------------------------------------------------------------- */
/* DFC — iblbm/ibm/dfc.py                                                     */
/* ------------------------------------------------------------------------- */

/* compute_lambda — dfc.py:126-186 */
void orc_dfc_lambda(int nx, int ny, int Lb, const double *Lx, const double *Ly, double rho_f,
                    double Larea, double dx, double dy, int delta_type, double *lambda_k)
{
    size_t N = (size_t)nx * ny;
    stencil_t *st = (stencil_t *)malloc(sizeof(stencil_t) * (size_t)(Lb > 0 ? Lb : 1));
    for (int l = 0; l < Lb; ++l) marker_stencil(Lx[l], Ly[l], dx, dy, nx, ny, delta_type, &st[l]);
    int S = Lb > 0 ? st[0].count : 0;
    double *Wt = (double *)calloc(N, sizeof(double));
    for (int k = 0; k < S; ++k)
        for (int l = 0; l < Lb; ++l) Wt[st[l].node[k]] += st[l].w[k];
    for (int l = 0; l < Lb; ++l) {
        double ws = 0.0;
        for (int k = 0; k < S; ++k) ws += Wt[st[l].node[k]] * st[l].w[k];
        lambda_k[l] = 1.0 / (2.0 * rho_f * Larea * ws);
    }
    free(Wt);
    free(st);
}

/* apply_dfc_correction CPU branch — dfc.py:256-342 (lines 321-342) with
 * interpolate_f (55-95), bounce_back_fi (98-123, rho_f = 1), spread_delta_f
 * (189-229).  fstar is corrected in place; dfc_force (Lb x 2) is the
 * distribution part of Tao (2019) Eq. (25) per marker. */
void orc_dfc_correction(int nx, int ny, int Lb, const double *Lx, const double *Ly,
                        const double *dvel, double *fstar, const double *lambda_k, double dx,
                        double dy, double Larea, int delta_type, double correction_scale,
                        double *dfc_force)
{
    size_t N = (size_t)nx * ny;
    stencil_t *st = (stencil_t *)malloc(sizeof(stencil_t) * (size_t)(Lb > 0 ? Lb : 1));
    for (int l = 0; l < Lb; ++l) marker_stencil(Lx[l], Ly[l], dx, dy, nx, ny, delta_type, &st[l]);
    int S = Lb > 0 ? st[0].count : 0;
    double *fi = (double *)calloc((size_t)Lb * 9, sizeof(double));
    double *dev = (double *)malloc(sizeof(double) * (size_t)Lb * 9);
    double *dfl = (double *)malloc(sizeof(double) * (size_t)Lb * 9);
    for (int k = 0; k < S; ++k)
        for (int l = 0; l < Lb; ++l) {
            long n = st[l].node[k];
            double w = st[l].w[k];
            for (int q = 0; q < 9; ++q) fi[9 * l + q] += fstar[9 * n + q] * w;
        }
    const double rho_f = 1.0, cs2 = 1.0 / 3.0;
    for (int l = 0; l < Lb; ++l) {
        for (int q = 0; q < 9; ++q) {
            double edu = e_dot(q, dvel[2 * l], dvel[2 * l + 1]);
            double fbb = fi[9 * l + OPP[q]] + 2.0 * W[q] * rho_f * edu / cs2;
            dev[9 * l + q] = fbb - fi[9 * l + q];
            dfl[9 * l + q] = correction_scale * lambda_k[l] * dev[9 * l + q];
        }
    }
    double *Ef = (double *)calloc(N * 9, sizeof(double));
    for (int k = 0; k < S; ++k)
        for (int l = 0; l < Lb; ++l) {
            long n = st[l].node[k];
            double w = st[l].w[k] * Larea;
            for (int q = 0; q < 9; ++q) Ef[9 * n + q] += dfl[9 * l + q] * w;
        }
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)(N * 9); ++k) fstar[k] = fstar[k] + Ef[k];
    for (int l = 0; l < Lb; ++l) {
        double sx = 0.0, sy = 0.0;
        for (int q = 0; q < 9; ++q) {
            double s = -(lambda_k[l] * dev[9 * l + q] * Larea);
            sx += s * (double)EX[q];
            sy += s * (double)EY[q];
        }
        dfc_force[2 * l] = correction_scale * sx;
        dfc_force[2 * l + 1] = correction_scale * sy;
    }
    free(Ef); free(fi); free(dev); free(dfl); free(st);
}

/* ------------------------------------------------------------------------- */
/* ||A||_inf for the MDF relaxation factor — iblbm/ibm/a_norm.py:75-172       */
/* (marker coordinates already in lattice units, dx = 1)                      */
/* ------------------------------------------------------------------------- */
double orc_a_norm_inf(int Lb, const double *Lx, const double *Ly, int delta_type, double Larea)
{
    const double dx = 1.0;
    int a = stencil_a(delta_type);
    double cutoff = 2.0 * a * dx;
    double factor = Larea / (dx * dx);
    double best = -INFINITY;
    for (int l = 0; l < Lb; ++l) {
        double acc = 0.0;
        for (int m = 0; m < Lb; ++m) {
            if (fabs(Lx[l] - Lx[m]) >= cutoff || fabs(Ly[l] - Ly[m]) >= cutoff) continue;
            double lo = fmax(Lx[l], Lx[m]) - a * dx, hi = fmin(Lx[l], Lx[m]) + a * dx;
            long i_lo = (long)ceil(lo / dx), i_hi = (long)floor(hi / dx) + 1;
            if (i_lo >= i_hi) continue;
            /* np.sum over a short vector (< 8 entries): sequential */
            double sx = 0.0;
            for (long i = i_lo; i < i_hi; ++i) {
                double x = (double)i * dx;
                sx += phi(delta_type, (x - Lx[l]) / dx) * phi(delta_type, (x - Lx[m]) / dx);
            }
            if (sx == 0.0) continue;
            lo = fmax(Ly[l], Ly[m]) - a * dx;
            hi = fmin(Ly[l], Ly[m]) + a * dx;
            long j_lo = (long)ceil(lo / dx), j_hi = (long)floor(hi / dx) + 1;
            if (j_lo >= j_hi) continue;
            double sy = 0.0;
            for (long j = j_lo; j < j_hi; ++j) {
                double y = (double)j * dx;
                sy += phi(delta_type, (y - Ly[l]) / dx) * phi(delta_type, (y - Ly[m]) / dx);
            }
            if (sy == 0.0) continue;
            acc += factor * sx * sy;
        }
        if (acc > best) best = acc;
    }
    return best;
}
