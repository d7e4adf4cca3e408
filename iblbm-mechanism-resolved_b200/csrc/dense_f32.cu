// dense_f32.cu — fused timestep in the FP32 shifted-population form.
//
// Same schedule as dense_f64.cu (pull-stream, closure, band correction,
// moments, velocity correction, equilibrium, collision, store) on deviations
// g = f - w held in FP32: 72 bytes per lattice update.  Compiled with the
// default multiply-add contraction.
#include <cstdint>
#include "shifted.cuh"

namespace iblbm {

void make_params32(const iblbm_case& c, CollParams32& cp, BcParams32& bc)
{
    cp.inv_tau = (float)(1.0 / c.tau);
    cp.guo_pref = (float)(1.0 - 0.5 / c.tau);
    cp.s_plus = (float)(1.0 / c.tau);
    cp.s_minus = (float)c.s_minus;
    cp.dt = (float)c.dt;
    for (int q = 0; q < 9; ++q) cp.S[q] = (float)c.S[q];
    bc.inflow_u = (float)c.inflow_u;
    bc.dens = (float)c.dens;
    const double u0 = c.inflow_u, u2 = u0 * u0;
    for (int q = 0; q < 9; ++q) {
        const double eU = (double)ex_(q) * u0;
        const double feq = c.dens * w_(q) * (1.0 + 3.0 * eU + 4.5 * eU * eU - 1.5 * u2);
        bc.geq_in[q] = (float)(feq - w_(q));
    }
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

// Four consecutive nodes per thread, one warp per 128-node row segment,
// blockDim.y rows per CTA.  Each population plane is read with one aligned
// 16-byte load per thread; the x-shifted pull sources come from the neighbouring
// lane's load (warp shuffle) or, at the warp's two ends, from one scalar load.
// Groups that touch the lattice boundary or the skipped box take the per-node
// path (closures, exact skip test).
__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__global__ void __launch_bounds__(256) dense32_vec4_kernel(const iblbm_dense32_args a, CollParams32 cp, BcParams32 bc)
{
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int lane = threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= g.ny) return;  // uniform over the warp
    const int i0 = (blockIdx.x * 32 + lane) * 4;
    int sx0 = 0, sy0 = 0, sx1 = -1, sy1 = -1;
    if (a.skip_box) {
        sx0 = __ldg(a.skip_box + 0);
        sy0 = __ldg(a.skip_box + 1);
        sx1 = sx0 + __ldg(a.skip_box + 2) - 1;
        sy1 = sy0 + __ldg(a.skip_box + 3) - 1;
    }
    const bool row_skip = j >= sy0 && j <= sy1;
    const bool interior_row = j >= 1 && j <= g.ny - 2;
    const bool fast = interior_row && i0 >= 4 && i0 + 3 <= g.nx - 2 && !(row_skip && i0 <= sx1 && i0 + 3 >= sx0);
    const BandView32 bv{a.band.box, a.band.map, a.band.fib, a.band.df};
    const DenseOut32 o{a.fpost_next, a.uring_next, OUT ? a.ro_out : nullptr, OUT ? a.U_out : nullptr,
                       OUT ? a.fstar_out : nullptr};
    float v[9][4];
    if (interior_row) {  // uniform over the warp: every lane takes part in the shuffles
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float* p = a.fpost_prev + q * g.qstride + (long long)(j - ey_(q)) * g.pitch;
            const float4 c = i0 < g.nx ? ld4(p + i0) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (ex_(q) == 0) {
                v[q][0] = c.x; v[q][1] = c.y; v[q][2] = c.z; v[q][3] = c.w;
            } else if (ex_(q) == 1) {  // source i - 1
                float left = __shfl_up_sync(0xffffffffu, c.w, 1);
                if (lane == 0) left = (i0 >= 1 && i0 <= g.nx) ? __ldg(p + i0 - 1) : 0.f;
                v[q][0] = left; v[q][1] = c.x; v[q][2] = c.y; v[q][3] = c.z;
            } else {  // source i + 1
                float right = __shfl_down_sync(0xffffffffu, c.x, 1);
                if (lane == 31) right = (i0 + 4 < g.nx) ? __ldg(p + i0 + 4) : 0.f;
                v[q][0] = c.y; v[q][1] = c.z; v[q][2] = c.w; v[q][3] = right;
            }
        }
    }
    if (fast) {
        float w[9][4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float f[9], out[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) f[q] = v[q][k];
            node_core32<COLL, BC, INCOMP, IBM, OUT>(f, g, cp, bv, o, i0 + k, j, out);
#pragma unroll
            for (int q = 0; q < 9; ++q) w[q][k] = out[q];
        }
        float* dst = a.fpost_next + (long long)j * g.pitch + i0;
#pragma unroll
        for (int q = 0; q < 9; ++q)
            *reinterpret_cast<float4*>(dst + q * g.qstride) = make_float4(w[q][0], w[q][1], w[q][2], w[q][3]);
    } else {
#pragma unroll 1
        for (int k = 0; k < 4; ++k) {
            const int i = i0 + k;
            if (i >= g.nx || (row_skip && i >= sx0 && i <= sx1)) continue;
            dense_node32<COLL, BC, INCOMP, IBM, OUT>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
        }
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
    if (a.tile_nodes == 1) {
        dim3 block(256, 1), grid((a.g.nx + 255) / 256, a.g.ny);
        if (out) dense32_kernel<COLL, BC, INCOMP, IBM, true><<<grid, block, 0, s>>>(a, cp, bc);
        else dense32_kernel<COLL, BC, INCOMP, IBM, false><<<grid, block, 0, s>>>(a, cp, bc);
        return cudaGetLastError();
    }
    const int rows = a.tile_rows > 0 ? a.tile_rows : 4;
    dim3 block(32, rows), grid((a.g.nx + 127) / 128, (a.g.ny + rows - 1) / rows);
    if (out) dense32_vec4_kernel<COLL, BC, INCOMP, IBM, true><<<grid, block, 0, s>>>(a, cp, bc);
    else dense32_vec4_kernel<COLL, BC, INCOMP, IBM, false><<<grid, block, 0, s>>>(a, cp, bc);
    return cudaGetLastError();
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
    if ((a->c.bc == BC_OPEN || a->c.bc == BC_VELOCITY_INLET) && (!a->uring_prev || !a->uring_next))
        return IBLBM_E_ARG;
    if (a->ibm != IBM_NONE && (!a->band.box || !a->band.map)) return IBLBM_E_ARG;
    if ((a->ibm == IBM_DF || a->ibm == IBM_MDF) && !a->band.fib) return IBLBM_E_ARG;
    if (a->ibm == IBM_DFC && !a->band.df) return IBLBM_E_ARG;
    if (a->skip_box && a->only_box) return IBLBM_E_ARG;
    if (a->tile_nodes != 0 && a->tile_nodes != 1 && a->tile_nodes != 4) return IBLBM_E_ARG;
    if (a->tile_rows < 0 || a->tile_rows > 8 || (a->tile_rows & (a->tile_rows - 1)) != 0) return IBLBM_E_ARG;
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
