// dense_node.cuh — the per-node FP64 timestep (pull-stream, closure, band
// correction, moments, velocity correction, equilibrium, collision, store),
// shared by the bulk kernel and the band kernel's box update.  Include from
// translation units compiled with -fmad=false.
#pragma once
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

__device__ __forceinline__ int band_lookup(const iblbm_band_view& bv, int nx, int i, int j)
{
    const int x0 = __ldg(bv.box + 0), y0 = __ldg(bv.box + 1), w = __ldg(bv.box + 2), h = __ldg(bv.box + 3);
    if (i < x0 || i >= x0 + w || j < y0 || j >= y0 + h) return -1;
    return bv.map[(long long)j * nx + i];
}

// BGK + Guo — iblbm/lbm/collision/bgk.py:25-40
template <bool INCOMP, bool FORCED>
__device__ __forceinline__ void collide_bgk(const double* f, double ro, double u0, double u1, double F0,
                                            double F1, const CollParams& cp, double* out)
{
    const double u2 = u0 * u0 + u1 * u1;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double fe = feq_q<INCOMP>(q, ro, u0, u1, u2);
        double v = f[q] - cp.inv_tau * (f[q] - fe);
        if (FORCED) {
            const double ex = (double)ex_(q), ey = (double)ey_(q);
            const double ax = ex - u0, ay = ey - u1;
            const double eU = ex * u0 + ey * u1;
            const double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
            const double F_ni = cp.guo_pref * w_(q) * term;
            v = v + F_ni * cp.dt;
        }
        out[q] = v;
    }
}

// TRT + Guo — iblbm/lbm/collision/trt.py:38-67
template <bool INCOMP, bool FORCED>
__device__ __forceinline__ void collide_trt(const double* f, double ro, double u0, double u1, double F0,
                                            double F1, const CollParams& cp, double* out)
{
    const double u2 = u0 * u0 + u1 * u1;
    double fe[9], bare[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) fe[q] = feq_q<INCOMP>(q, ro, u0, u1, u2);
    if (FORCED) {
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const double ex = (double)ex_(q), ey = (double)ey_(q);
            const double ax = ex - u0, ay = ey - u1;
            const double eU = ex * u0 + ey * u1;
            const double term = ((3.0 * ax + 9.0 * eU * ex) * F0 + (3.0 * ay + 9.0 * eU * ey) * F1);
            bare[q] = w_(q) * term;
        }
    }
    const double gp = 1.0 - 0.5 * cp.s_plus, gm = 1.0 - 0.5 * cp.s_minus;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int o = opp_(q);
        const double fp = 0.5 * (f[q] + f[o]);
        const double fm = 0.5 * (f[q] - f[o]);
        const double ep = 0.5 * (fe[q] + fe[o]);
        const double em = 0.5 * (fe[q] - fe[o]);
        const double coll = (cp.s_plus * (fp - ep) + cp.s_minus * (fm - em));
        double v = f[q] - coll;
        if (FORCED) {
            const double bp = 0.5 * (bare[q] + bare[o]);
            const double bm = 0.5 * (bare[q] - bare[o]);
            const double F_ni = gp * bp + gm * bm;
            v = v + F_ni * cp.dt;
        }
        out[q] = v;
    }
}

// Central-moment MRT + Guo — iblbm/lbm/collision/cm_mrt.py:52-165
template <bool FORCED>
__device__ __forceinline__ void collide_cmmrt(const double* f, double ux, double uy, double F0, double F1,
                                              const CollParams& cp, double* out)
{
    double cm0 = 0.0, cm1 = 0.0, cm2 = 0.0, cm3 = 0.0, cm4 = 0.0, cm5 = 0.0, cm6 = 0.0, cm7 = 0.0, cm8 = 0.0;
    double Fc0 = 0.0, Fc1 = 0.0, Fc2 = 0.0, Fc3 = 0.0, Fc4 = 0.0, Fc5 = 0.0, Fc6 = 0.0, Fc7 = 0.0, Fc8 = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double val = f[q];
        const double ex = (double)ex_(q), ey = (double)ey_(q);
        const double cix = ex - ux, ciy = ey - uy;
        const double cix2 = cix * cix, ciy2 = ciy * ciy;
        cm0 += val;
        cm1 += val * cix;
        cm2 += val * ciy;
        cm3 += val * cix2;
        cm4 += val * ciy2;
        cm5 += val * cix * ciy;
        cm6 += val * cix2 * ciy;
        cm7 += val * cix * ciy2;
        cm8 += val * cix2 * ciy2;
        if (FORCED) {
            const double eU = ex * ux + ey * uy;
            const double term = ((3.0 * cix + 9.0 * eU * ex) * F0 + (3.0 * ciy + 9.0 * eU * ey) * F1);
            const double Fb = w_(q) * term;
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
    }
    const double* S = cp.S;
    const double rho = cm0, cs2 = 1.0 / 3.0, cs4 = 1.0 / 9.0, dt = cp.dt;
    double cp0 = cm0 - S[0] * (cm0 - rho);
    double cp1 = cm1 - S[1] * (cm1 - 0.0);
    double cp2 = cm2 - S[2] * (cm2 - 0.0);
    double cp3 = cm3 - S[3] * (cm3 - rho * cs2);
    double cp4 = cm4 - S[4] * (cm4 - rho * cs2);
    double cp5 = cm5 - S[5] * (cm5 - 0.0);
    double cp6 = cm6 - S[6] * (cm6 - 0.0);
    double cp7 = cm7 - S[7] * (cm7 - 0.0);
    double cp8 = cm8 - S[8] * (cm8 - rho * cs4);
    if (FORCED) {
        cp0 = cp0 + (1.0 - 0.5 * S[0]) * Fc0 * dt;
        cp1 = cp1 + (1.0 - 0.5 * S[1]) * Fc1 * dt;
        cp2 = cp2 + (1.0 - 0.5 * S[2]) * Fc2 * dt;
        cp3 = cp3 + (1.0 - 0.5 * S[3]) * Fc3 * dt;
        cp4 = cp4 + (1.0 - 0.5 * S[4]) * Fc4 * dt;
        cp5 = cp5 + (1.0 - 0.5 * S[5]) * Fc5 * dt;
        cp6 = cp6 + (1.0 - 0.5 * S[6]) * Fc6 * dt;
        cp7 = cp7 + (1.0 - 0.5 * S[7]) * Fc7 * dt;
        cp8 = cp8 + (1.0 - 0.5 * S[8]) * Fc8 * dt;
    }
    const double ux2 = ux * ux, uy2 = uy * uy;
    const double k0 = cp0;
    const double k1 = cp1 + ux * cp0;
    const double k2 = cp2 + uy * cp0;
    const double k3 = cp3 + 2.0 * ux * cp1 + ux2 * cp0;
    const double k4 = cp4 + 2.0 * uy * cp2 + uy2 * cp0;
    const double k5 = cp5 + uy * cp1 + ux * cp2 + ux * uy * cp0;
    const double k6 = (cp6 + uy * cp3 + 2.0 * ux * cp5 + 2.0 * ux * uy * cp1 + ux2 * cp2 + ux2 * uy * cp0);
    const double k7 = (cp7 + 2.0 * uy * cp5 + ux * cp4 + 2.0 * ux * uy * cp2 + uy2 * cp1 + ux * uy2 * cp0);
    const double k8 = (cp8 + 2.0 * uy * cp6 + uy2 * cp3 + 2.0 * ux * cp7 + 4.0 * ux * uy * cp5 +
                       2.0 * ux * uy2 * cp1 + ux2 * cp4 + 2.0 * ux2 * uy * cp2 + ux2 * uy2 * cp0);
    out[0] = k0 - k3 - k4 + k8;
    out[1] = 0.5 * (k1 + k3 - k7 - k8);
    out[2] = 0.5 * (k2 + k4 - k6 - k8);
    out[3] = 0.5 * (-k1 + k3 + k7 - k8);
    out[4] = 0.5 * (-k2 + k4 + k6 - k8);
    out[5] = 0.25 * (k5 + k6 + k7 + k8);
    out[6] = 0.25 * (-k5 + k6 - k7 + k8);
    out[7] = 0.25 * (k5 - k6 - k7 + k8);
    out[8] = 0.25 * (-k5 - k6 + k7 + k8);
}

template <int COLL, bool INCOMP, bool FORCED>
__device__ __forceinline__ void collide(const double* f, double ro, double u0, double u1, double F0, double F1,
                                        const CollParams& cp, double* out)
{
    if (COLL == COLL_BGK) collide_bgk<INCOMP, FORCED>(f, ro, u0, u1, F0, F1, cp, out);
    else if (COLL == COLL_TRT) collide_trt<INCOMP, FORCED>(f, ro, u0, u1, F0, F1, cp, out);
    else collide_cmmrt<FORCED>(f, u0, u1, F0, F1, cp, out);
}


struct DenseOut {
    double* fpost_next;
    double* uring_next;
    double* ro_out;
    double* U_out;
    double* fstar_out;
};

template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__device__ __forceinline__ void dense_node(const double* __restrict__ fpost_prev, const double* __restrict__ uring_prev,
                                           const Geom& g, const CollParams& cp, const BcParams& bc,
                                           const iblbm_band_view& band, const DenseOut& o, int i, int j)
{
    double f[9];
    fstar_node<BC>(fpost_prev, uring_prev, g, bc, INCOMP, i, j, f);
    int b = -1;
    if (IBM != IBM_NONE) b = band_lookup(band, g.nx, i, j);
    if (IBM == IBM_DFC && b >= 0) {
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = f[q] + band.df[9 * (long long)b + q];
    }
    const long long site = (long long)j * g.pitch + i;
    if (OUT && o.fstar_out) {
#pragma unroll
        for (int q = 0; q < 9; ++q) o.fstar_out[q * g.qstride + site] = f[q];
    }
    double ro, u0, u1;
    macro_seq(f, INCOMP, ro, u0, u1);
    double out[9];
    if ((IBM == IBM_DF || IBM == IBM_MDF) && b >= 0) {
        // iblbm/ibm/dispatch.py:18-33 (CPU branch)
        const double F0 = band.fib[2 * (long long)b], F1 = band.fib[2 * (long long)b + 1];
        if (INCOMP) {
            u0 = u0 + 0.5 * F0 * cp.dt;
            u1 = u1 + 0.5 * F1 * cp.dt;
        } else {
            u0 = u0 + F0 * cp.dt / (2.0 * ro);
            u1 = u1 + F1 * cp.dt / (2.0 * ro);
        }
        collide<COLL, INCOMP, true>(f, ro, u0, u1, F0, F1, cp, out);
    } else {
        collide<COLL, INCOMP, false>(f, ro, u0, u1, 0.0, 0.0, cp, out);
    }
    if (OUT) {
        const long long n = (long long)j * g.nx + i;
        if (o.ro_out) o.ro_out[n] = ro;
        if (o.U_out) { o.U_out[2 * n] = u0; o.U_out[2 * n + 1] = u1; }
    }
    if ((BC == BC_OPEN || BC == BC_VELOCITY_INLET) && is_ring(g, i, j)) {
        const long long n = (long long)j * g.nx + i;
        o.uring_next[2 * n] = u0;
        o.uring_next[2 * n + 1] = u1;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) o.fpost_next[q * g.qstride + site] = out[q];
}

}  // namespace iblbm
