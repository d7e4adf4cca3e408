// dense_f64.cu — fused FP64 timestep over the whole lattice.
//
// One thread per node: pull-stream the nine populations from the previous
// post-collision buffer, apply the boundary closure on edge nodes, add the DFC
// correction on band nodes, take the moments, apply the Guo half-force velocity
// correction on band nodes, build the equilibrium and collide (BGK / TRT /
// CM-MRT), and store the nine post-collision populations.  This replaces the
// reference's chain of dense passes (collide, stream, boundary, macroscopic,
// IBM correction, feq) with one read and one write of the populations per
// step: 144 bytes per lattice update in FP64.
//
// Compiled with -fmad=false: the arithmetic is the reference CPU path's,
// operation for operation (see common.cuh).
#include "common.cuh"
#include "../../include/iblbm_b200.h"

#include "dense_node.cuh"

namespace iblbm {

template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__global__ void __launch_bounds__(128) dense_step_kernel(const iblbm_dense_args a, CollParams cp, BcParams bc)
{
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= g.nx) return;
    if (a.skip_box) {
        // nodes inside the skip box are updated by the band kernel of this step
        const int x0 = __ldg(a.skip_box + 0), y0 = __ldg(a.skip_box + 1);
        const int w = __ldg(a.skip_box + 2), h = __ldg(a.skip_box + 3);
        if (i >= x0 && i < x0 + w && j >= y0 && j < y0 + h) return;
    }
    DenseOut o{a.fpost_next, a.uring_next, OUT ? a.ro_out : nullptr, OUT ? a.U_out : nullptr,
               OUT ? a.fstar_out : nullptr};
    dense_node<COLL, BC, INCOMP, IBM, OUT>(a.fpost_prev, a.uring_prev, g, cp, bc, a.band, o, i, j);
}

// Box pass: the nodes of a small box (read from device memory, so one launch
// shape serves every step of a moving body), grid-stride over its cells.
template <int COLL, int BC, bool INCOMP, int IBM, bool OUT>
__global__ void __launch_bounds__(128) dense_box_kernel(const iblbm_dense_args a, CollParams cp, BcParams bc)
{
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int x0 = __ldg(a.only_box + 0), y0 = __ldg(a.only_box + 1);
    const int w = __ldg(a.only_box + 2), h = __ldg(a.only_box + 3);
    const int cells = w * h;
    DenseOut o{a.fpost_next, a.uring_next, OUT ? a.ro_out : nullptr, OUT ? a.U_out : nullptr,
               OUT ? a.fstar_out : nullptr};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
        const int i = x0 + c % w, j = y0 + c / w;
        if (i < 0 || i >= g.nx || j < 0 || j >= g.ny) continue;
        dense_node<COLL, BC, INCOMP, IBM, OUT>(a.fpost_prev, a.uring_prev, g, cp, bc, a.band, o, i, j);
    }
}

template <int COLL, int BC, bool INCOMP, int IBM>
static cudaError_t launch_ibm(const iblbm_dense_args& a, const CollParams& cp, const BcParams& bc, cudaStream_t s)
{
    const bool out = a.ro_out || a.U_out || a.fstar_out;
    if (a.only_box) {
        const int nblk = a.box_blocks > 0 ? a.box_blocks : 64;
        if (out) dense_box_kernel<COLL, BC, INCOMP, IBM, true><<<nblk, 128, 0, s>>>(a, cp, bc);
        else dense_box_kernel<COLL, BC, INCOMP, IBM, false><<<nblk, 128, 0, s>>>(a, cp, bc);
        return cudaGetLastError();
    }
    dim3 block(128, 1), grid((a.g.nx + 127) / 128, a.g.ny);
    if (out) dense_step_kernel<COLL, BC, INCOMP, IBM, true><<<grid, block, 0, s>>>(a, cp, bc);
    else dense_step_kernel<COLL, BC, INCOMP, IBM, false><<<grid, block, 0, s>>>(a, cp, bc);
    return cudaGetLastError();
}

template <int COLL, int BC, bool INCOMP>
static cudaError_t launch_inc(const iblbm_dense_args& a, const CollParams& cp, const BcParams& bc, cudaStream_t s)
{
    switch (a.ibm) {
    case IBM_NONE: return launch_ibm<COLL, BC, INCOMP, IBM_NONE>(a, cp, bc, s);
    case IBM_DF: return launch_ibm<COLL, BC, INCOMP, IBM_DF>(a, cp, bc, s);
    case IBM_MDF: return launch_ibm<COLL, BC, INCOMP, IBM_MDF>(a, cp, bc, s);
    case IBM_DFC: return launch_ibm<COLL, BC, INCOMP, IBM_DFC>(a, cp, bc, s);
    }
    return cudaErrorInvalidValue;
}

template <int COLL, int BC>
static cudaError_t launch_bc(const iblbm_dense_args& a, const CollParams& cp, const BcParams& bc, cudaStream_t s)
{
    return a.c.incompressible ? launch_inc<COLL, BC, true>(a, cp, bc, s) : launch_inc<COLL, BC, false>(a, cp, bc, s);
}

template <int COLL>
static cudaError_t launch_coll(const iblbm_dense_args& a, const CollParams& cp, const BcParams& bc, cudaStream_t s)
{
    switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN: return launch_bc<COLL, BC_DIRICHLET_NEUMANN>(a, cp, bc, s);
    case BC_OPEN: return launch_bc<COLL, BC_OPEN>(a, cp, bc, s);
    case BC_SETTLING: return launch_bc<COLL, BC_SETTLING>(a, cp, bc, s);
    case BC_VELOCITY_INLET: return launch_bc<COLL, BC_VELOCITY_INLET>(a, cp, bc, s);
    case BC_TG: return launch_bc<COLL, BC_TG>(a, cp, bc, s);
    }
    return cudaErrorInvalidValue;
}

// Host-side parameter derivation, with the reference's formulas.
void make_params(const iblbm_case& c, CollParams& cp, BcParams& bc)
{
    cp.tau = c.tau;
    cp.inv_tau = 1.0 / c.tau;        // bgk.py:28
    cp.guo_pref = 1.0 - 0.5 / c.tau; // bgk.py:29
    cp.s_plus = 1.0 / c.tau;         // trt.py:84
    cp.s_minus = c.s_minus;
    for (int q = 0; q < 9; ++q) cp.S[q] = c.S[q];
    cp.dt = c.dt;
    make_bc(c, bc);
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_dense_step_f64(const iblbm_dense_args* a, void* stream)
{
    if (!a || !a->fpost_prev || !a->fpost_next || a->g.nx < 4 || a->g.ny < 4 || a->g.pitch < a->g.nx)
        return IBLBM_E_ARG;
    if ((a->c.bc == BC_OPEN || a->c.bc == BC_VELOCITY_INLET) && (!a->uring_prev || !a->uring_next))
        return IBLBM_E_ARG;
    if (a->ibm != IBM_NONE && (!a->band.box || !a->band.map)) return IBLBM_E_ARG;
    if (a->c.bc == BC_TG && (!a->c.tg_face || !a->c.tg_decay)) return IBLBM_E_ARG;
    if (a->skip_box && a->only_box) return IBLBM_E_ARG;
    if ((a->ibm == IBM_DF || a->ibm == IBM_MDF) && !a->band.fib) return IBLBM_E_ARG;
    if (a->ibm == IBM_DFC && !a->band.df) return IBLBM_E_ARG;
    CollParams cp;
    BcParams bc;
    make_params(a->c, cp, bc);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    switch (a->c.collision) {
    case COLL_BGK: e = launch_coll<COLL_BGK>(*a, cp, bc, s); break;
    case COLL_TRT: e = launch_coll<COLL_TRT>(*a, cp, bc, s); break;
    case COLL_CMMRT: e = launch_coll<COLL_CMMRT>(*a, cp, bc, s); break;
    default: return IBLBM_E_ARG;
    }
    return e == cudaSuccess ? IBLBM_OK : (e == cudaErrorInvalidValue ? IBLBM_E_ARG : IBLBM_E_LAUNCH);
}
