// dense_f32.cu — fused timestep in the FP32 shifted-population form.
//
// Same schedule as dense_f64.cu (pull-stream, closure, band correction,
// moments, velocity correction, equilibrium, collision, store) on deviations
// g = f - w held in FP32: 72 bytes per lattice update.  Compiled with the
// default multiply-add contraction.
#include <cstdint>
#include "shifted.cuh"

namespace iblbm {

cudaError_t launch_pipe32(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s);

void make_params32(const iblbm_case& c, CollParams32& cp, BcParams32& bc)
{
    cp.inv_tau = (float)(1.0 / c.tau);
    cp.guo_pref = (float)(1.0 - 0.5 / c.tau);
    cp.s_plus = (float)(1.0 / c.tau);
    cp.s_minus = (float)c.s_minus;
    cp.dt = (float)c.dt;
    for (int q = 0; q < 9; ++q) cp.S[q] = (float)c.S[q];
    make_bc(c, bc);
}

template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__global__ void __launch_bounds__(256) dense32_kernel(const iblbm_dense32_args a, CollParams32 cp, BcParams32 bc)
{
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= g.nx) return;
    if (a.skip_box) {
        const int x0 = __ldg(a.skip_box + 0), y0 = __ldg(a.skip_box + 1);
        const int w = __ldg(a.skip_box + 2), h = __ldg(a.skip_box + 3);
        if (i >= x0 && i < x0 + w && j >= y0 && j < y0 + h) return;
    }
    const BandView32 bv{a.band.box, a.band.map, a.band.fib, a.band.df};
    const DenseOut32 o{a.fpost_next, a.uring_next, OUT ? a.ro_out : nullptr, OUT ? a.U_out : nullptr,
                       OUT ? a.fstar_out : nullptr};
    dense_node32<COLL, BC, INCOMP, IBM, OUT>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
}

// NR nodes per thread, stacked in y: the 9 * NR pull loads of all of them are
// issued before the first collision, so each thread keeps NR times the bytes in
// flight of the one-node form (the pass is bound by outstanding loads, not by
// arithmetic).  128 threads per CTA along x, NR rows per CTA.
template <int COLL, int BC, bool INCOMP, int IBM, int NR>
__global__ void __launch_bounds__(128) dense32_rows_kernel(const iblbm_dense32_args a, CollParams32 cp, BcParams32 bc)
{
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j0 = blockIdx.y * NR;
    if (i >= g.nx) return;
    int sx0 = 0, sy0 = 0, sx1 = -1, sy1 = -1;
    if (a.skip_box) {
        sx0 = __ldg(a.skip_box + 0);
        sy0 = __ldg(a.skip_box + 1);
        sx1 = sx0 + __ldg(a.skip_box + 2) - 1;
        sy1 = sy0 + __ldg(a.skip_box + 3) - 1;
    }
    const bool col_skip = i >= sx0 && i <= sx1;
    int off[9];
    pull_offsets(g, off);
    float f[NR][9];
#pragma unroll
    for (int n = 0; n < NR; ++n)
        if (j0 + n < g.ny) pull_node(a.fpost_prev, g, off, i, j0 + n, f[n]);
    const BandView32 bv{a.band.box, a.band.map, a.band.fib, a.band.df};
    const DenseOut32 o{a.fpost_next, a.uring_next, nullptr, nullptr, nullptr};
#pragma unroll
    for (int n = 0; n < NR; ++n) {
        const int j = j0 + n;
        if (j >= g.ny || (col_skip && j >= sy0 && j <= sy1)) continue;
        closure_node<BC>(a.fpost_prev, a.uring_prev, g, bc, INCOMP, i, j, f[n]);
        float out[9];
        node_core32<COLL, has_ring<BC>(), INCOMP, IBM, false>(f[n], g, cp, bv, o, i, j, out);
        float* dst = a.fpost_next + (long long)j * g.pitch + i;
#pragma unroll
        for (int q = 0; q < 9; ++q) dst[q * g.qstride] = out[q];
    }
}

template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__global__ void __launch_bounds__(128) dense32_box_kernel(const iblbm_dense32_args a, CollParams32 cp, BcParams32 bc)
{
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int x0 = __ldg(a.only_box + 0), y0 = __ldg(a.only_box + 1);
    const int w = __ldg(a.only_box + 2), h = __ldg(a.only_box + 3);
    const BandView32 bv{a.band.box, a.band.map, a.band.fib, a.band.df};
    const DenseOut32 o{a.fpost_next, a.uring_next, OUT ? a.ro_out : nullptr, OUT ? a.U_out : nullptr,
                       OUT ? a.fstar_out : nullptr};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w * h; c += gridDim.x * blockDim.x) {
        const int i = x0 + c % w, j = y0 + c / w;
        if (i < 0 || i >= g.nx || j < 0 || j >= g.ny) continue;
        dense_node32<COLL, BC, INCOMP, IBM, OUT>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
    }
}

template <int COLL, int BC, bool INCOMP, int IBM>
static cudaError_t launch32_ibm(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    const bool out = a.ro_out || a.U_out || a.fstar_out;
    if (a.only_box) {
        const int nblk = a.box_blocks > 0 ? a.box_blocks : 64;
        if (out) dense32_box_kernel<COLL, BC, INCOMP, IBM, true><<<nblk, 128, 0, s>>>(a, cp, bc);
        else dense32_box_kernel<COLL, BC, INCOMP, IBM, false><<<nblk, 128, 0, s>>>(a, cp, bc);
        return cudaGetLastError();
    }
    if (out || a.tile == IBLBM_TILE_NODE) {
        dim3 block(256, 1), grid((a.g.nx + 255) / 256, a.g.ny);
        if (out) dense32_kernel<COLL, BC, INCOMP, IBM, true><<<grid, block, 0, s>>>(a, cp, bc);
        else dense32_kernel<COLL, BC, INCOMP, IBM, false><<<grid, block, 0, s>>>(a, cp, bc);
        return cudaGetLastError();
    }
    if (a.tile == IBLBM_TILE_ROWS2 || a.tile == IBLBM_TILE_ROWS4) {
        const int nr = a.tile == IBLBM_TILE_ROWS2 ? 2 : 4;
        dim3 grid((a.g.nx + 127) / 128, (a.g.ny + nr - 1) / nr);
        if (nr == 2) dense32_rows_kernel<COLL, BC, INCOMP, IBM, 2><<<grid, 128, 0, s>>>(a, cp, bc);
        else dense32_rows_kernel<COLL, BC, INCOMP, IBM, 4><<<grid, 128, 0, s>>>(a, cp, bc);
        return cudaGetLastError();
    }
    return launch_pipe32(a, cp, bc, s);
}

template <int COLL, int BC, bool INCOMP>
static cudaError_t launch32_inc(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    switch (a.ibm) {
    case IBM_NONE: return launch32_ibm<COLL, BC, INCOMP, IBM_NONE>(a, cp, bc, s);
    case IBM_DF: return launch32_ibm<COLL, BC, INCOMP, IBM_DF>(a, cp, bc, s);
    case IBM_MDF: return launch32_ibm<COLL, BC, INCOMP, IBM_MDF>(a, cp, bc, s);
    case IBM_DFC: return launch32_ibm<COLL, BC, INCOMP, IBM_DFC>(a, cp, bc, s);
    }
    return cudaErrorInvalidValue;
}

template <int COLL, int BC>
static cudaError_t launch32_bc(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    return a.c.incompressible ? launch32_inc<COLL, BC, true>(a, cp, bc, s) : launch32_inc<COLL, BC, false>(a, cp, bc, s);
}

template <int COLL>
static cudaError_t launch32_coll(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN: return launch32_bc<COLL, BC_DIRICHLET_NEUMANN>(a, cp, bc, s);
    case BC_OPEN: return launch32_bc<COLL, BC_OPEN>(a, cp, bc, s);
    case BC_SETTLING: return launch32_bc<COLL, BC_SETTLING>(a, cp, bc, s);
    case BC_VELOCITY_INLET: return launch32_bc<COLL, BC_VELOCITY_INLET>(a, cp, bc, s);
    case BC_TG: return launch32_bc<COLL, BC_TG>(a, cp, bc, s);
    }
    return cudaErrorInvalidValue;
}

// f (FP64, AoS) -> g = f - w (FP32, pitched SoA) and back
__global__ void to_shifted_kernel(const double* __restrict__ aos, Geom g, float* __restrict__ soa)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= g.nx) return;
    const long long n = (long long)j * g.nx + i;
#pragma unroll
    for (int q = 0; q < 9; ++q) soa[q * g.qstride + (long long)j * g.pitch + i] = (float)(aos[9 * n + q] - w_(q));
}

__global__ void from_shifted_kernel(const float* __restrict__ soa, Geom g, double* __restrict__ aos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= g.nx) return;
    const long long n = (long long)j * g.nx + i;
#pragma unroll
    for (int q = 0; q < 9; ++q) aos[9 * n + q] = (double)soa[q * g.qstride + (long long)j * g.pitch + i] + w_(q);
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_dense_step_f32(const iblbm_dense32_args* a, void* stream)
{
    if (!a || !a->fpost_prev || !a->fpost_next || a->g.nx < 4 || a->g.ny < 4 || a->g.pitch < a->g.nx)
        return IBLBM_E_ARG;
    if (9LL * a->g.qstride >= (1LL << 31)) return IBLBM_E_CAPACITY;  // 32-bit pull offsets
    if ((a->c.bc == BC_OPEN || a->c.bc == BC_VELOCITY_INLET) && (!a->uring_prev || !a->uring_next))
        return IBLBM_E_ARG;
    if (a->ibm != IBM_NONE && (!a->band.box || !a->band.map)) return IBLBM_E_ARG;
    if ((a->ibm == IBM_DF || a->ibm == IBM_MDF) && !a->band.fib) return IBLBM_E_ARG;
    if (a->ibm == IBM_DFC && !a->band.df) return IBLBM_E_ARG;
    if (a->c.bc == BC_TG && (!a->c.tg_face || !a->c.tg_decay)) return IBLBM_E_ARG;
    if (a->skip_box && a->only_box) return IBLBM_E_ARG;
    if (a->tile < IBLBM_TILE_PIPE_4x2 || a->tile > IBLBM_TILE_ROWS4) return IBLBM_E_ARG;
    if ((reinterpret_cast<uintptr_t>(a->fpost_prev) & 15) || (reinterpret_cast<uintptr_t>(a->fpost_next) & 15) ||
        (a->g.pitch & 3))
        return IBLBM_E_ARG;
    CollParams32 cp;
    BcParams32 bc;
    make_params32(a->c, cp, bc);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    switch (a->c.collision) {
    case COLL_BGK: e = launch32_coll<COLL_BGK>(*a, cp, bc, s); break;
    case COLL_TRT: e = launch32_coll<COLL_TRT>(*a, cp, bc, s); break;
    case COLL_CMMRT: e = launch32_coll<COLL_CMMRT>(*a, cp, bc, s); break;
    default: return IBLBM_E_ARG;
    }
    return e == cudaSuccess ? IBLBM_OK : (e == cudaErrorInvalidValue ? IBLBM_E_ARG : IBLBM_E_LAUNCH);
}

extern "C" int iblbm_to_shifted_f32(const double* aos, iblbm_geom g, float* soa, void* s)
{
    if (!aos || !soa || g.nx < 1 || g.ny < 1 || g.pitch < g.nx) return IBLBM_E_ARG;
    dim3 grid((g.nx + 127) / 128, g.ny);
    to_shifted_kernel<<<grid, 128, 0, (cudaStream_t)s>>>(aos, Geom{g.nx, g.ny, g.pitch, g.qstride}, soa);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

extern "C" int iblbm_from_shifted_f32(const float* soa, iblbm_geom g, double* aos, void* s)
{
    if (!aos || !soa || g.nx < 1 || g.ny < 1 || g.pitch < g.nx) return IBLBM_E_ARG;
    dim3 grid((g.nx + 127) / 128, g.ny);
    from_shifted_kernel<<<grid, 128, 0, (cudaStream_t)s>>>(soa, Geom{g.nx, g.ny, g.pitch, g.qstride}, aos);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

