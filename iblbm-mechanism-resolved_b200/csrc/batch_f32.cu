// batch_f32.cu — batched FP32 collide-stream pass over many independent cases.
// Split from dense_f32.cu so the units compile in parallel.
#include <cstdint>
#include "shifted.cuh"

namespace iblbm {

void make_params32(const iblbm_case& c, CollParams32& cp, BcParams32& bc);

// ---------------------------------------------------------------------------
// Batched pass: many independent cases of one kind (collision, closure,
// compressibility, band method) in one launch.  The per-case geometry,
// pointers and rounded parameters travel in the kernel's parameter block
// (read through the constant cache); CTA b finds its case by binary search over
// the cases' block offsets, then runs the multi-row node pass (NR nodes per
// thread) on its part of that case's lattice.  Cases of uneven size cost only
// their own blocks.
// ---------------------------------------------------------------------------
constexpr int BATCH_MAX = 72;

struct BatchCase {
    int nx, ny, pitch, bx;   // bx: 128-node column blocks
    int kind;                // collision * 8 + closure * 2 + incompressible (mixed bulk launches)
    long long qstride;
    const float* fp;
    float* fn;
    const float* urp;
    float* urn;
    const int* box;
    const int* map;
    const float* fib;
    const float* df;
    const int* skip_box;
    const int* only_box;
    CollParams32 cp;
    BcParams32 bc;
};

struct BatchTable {
    int n;
    int off[BATCH_MAX + 1];
    BatchCase c[BATCH_MAX];
};

__device__ __forceinline__ int batch_case(const BatchTable& t, int blk)
{
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.off[mid] <= blk) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// NR nodes per thread stacked in y on block `local` of case c.
template <int COLL, int BC, bool INCOMP, int IBM, int NR>
__device__ __forceinline__ void batch_rows(const BatchCase& c, int local)
{
    const Geom g{c.nx, c.ny, c.pitch, c.qstride};
    const int i = (local % c.bx) * 128 + threadIdx.x;
    const int j0 = (local / c.bx) * NR;
    if (i >= g.nx) return;
    int sx0 = 0, sy0 = 0, sx1 = -1, sy1 = -1;
    if (c.skip_box) {
        sx0 = __ldg(c.skip_box + 0);
        sy0 = __ldg(c.skip_box + 1);
        sx1 = sx0 + __ldg(c.skip_box + 2) - 1;
        sy1 = sy0 + __ldg(c.skip_box + 3) - 1;
    }
    const bool col_skip = i >= sx0 && i <= sx1;
    int off[9];
    pull_offsets(g, off);
    float f[NR][9];
#pragma unroll
    for (int n = 0; n < NR; ++n)
        if (j0 + n < g.ny) pull_node(c.fp, g, off, i, j0 + n, f[n]);
    const BandView32 bv{c.box, c.map, c.fib, c.df};
    const DenseOut32 o{c.fn, c.urn, nullptr, nullptr, nullptr};
#pragma unroll
    for (int n = 0; n < NR; ++n) {
        const int j = j0 + n;
        if (j >= g.ny || (col_skip && j >= sy0 && j <= sy1)) continue;
        closure_node<BC>(c.fp, c.urp, g, c.bc, INCOMP, i, j, f[n]);
        float out[9];
        node_core32<COLL, has_ring<BC>(), INCOMP, IBM, false>(f[n], g, c.cp, bv, o, i, j, out);
        float* dst = c.fn + (long long)j * g.pitch + i;
#pragma unroll
        for (int q = 0; q < 9; ++q) dst[q * g.qstride] = out[q];
    }
}

// Ten resident CTAs per SM (at most 51 registers a thread; 48 are used): more
// loads in flight per SM than the 56-60 registers the kinds take unbounded.
// Over the 72-case sweep the bulk passes took 0.757 ms per step this way
// against 0.771-0.774 ms (the small spills it costs stay in L1); a bound of 12
// CTAs (40 registers) spills more and lost the gain.
template <int COLL, int BC, bool INCOMP, int IBM, int NR>
__global__ void __launch_bounds__(128, 10) dense32_batch_kernel(const __grid_constant__ BatchTable t)
{
    const int ci = batch_case(t, blockIdx.x);
    batch_rows<COLL, BC, INCOMP, IBM, NR>(t.c[ci], blockIdx.x - t.off[ci]);
}

// Bulk passes (no band) of cases of different kinds in one launch: each CTA
// dispatches on its case's kind, so the launch has one tail instead of one per
// kind.
template <int COLL, int NR>
__device__ __forceinline__ void batch_rows_bc(const BatchCase& c, int local, int bcv, bool inc)
{
    switch (bcv) {
    case BC_DIRICHLET_NEUMANN:
        if (inc) batch_rows<COLL, BC_DIRICHLET_NEUMANN, true, IBM_NONE, NR>(c, local);
        else batch_rows<COLL, BC_DIRICHLET_NEUMANN, false, IBM_NONE, NR>(c, local);
        break;
    case BC_OPEN:
        if (inc) batch_rows<COLL, BC_OPEN, true, IBM_NONE, NR>(c, local);
        else batch_rows<COLL, BC_OPEN, false, IBM_NONE, NR>(c, local);
        break;
    case BC_SETTLING:
        if (inc) batch_rows<COLL, BC_SETTLING, true, IBM_NONE, NR>(c, local);
        else batch_rows<COLL, BC_SETTLING, false, IBM_NONE, NR>(c, local);
        break;
    default:
        if (inc) batch_rows<COLL, BC_VELOCITY_INLET, true, IBM_NONE, NR>(c, local);
        else batch_rows<COLL, BC_VELOCITY_INLET, false, IBM_NONE, NR>(c, local);
        break;
    }
}

template <int NR>
__global__ void __launch_bounds__(128) dense32_batch_mixed_kernel(const __grid_constant__ BatchTable t)
{
    const int ci = batch_case(t, blockIdx.x);
    const BatchCase& c = t.c[ci];
    const int local = blockIdx.x - t.off[ci];
    const int coll = c.kind >> 3, bcv = (c.kind >> 1) & 3;
    const bool inc = (c.kind & 1) != 0;
    if (coll == COLL_BGK) batch_rows_bc<COLL_BGK, NR>(c, local, bcv, inc);
    else if (coll == COLL_TRT) batch_rows_bc<COLL_TRT, NR>(c, local, bcv, inc);
    else batch_rows_bc<COLL_CMMRT, NR>(c, local, bcv, inc);
}

// Box passes of a batch: blockIdx.y is the case, grid-stride over its box.
template <int COLL, int BC, bool INCOMP, int IBM>
__global__ void __launch_bounds__(128) dense32_box_batch_kernel(const __grid_constant__ BatchTable t)
{
    const BatchCase& c = t.c[blockIdx.y];
    const Geom g{c.nx, c.ny, c.pitch, c.qstride};
    const int x0 = __ldg(c.only_box + 0), y0 = __ldg(c.only_box + 1);
    const int w = __ldg(c.only_box + 2), h = __ldg(c.only_box + 3);
    const BandView32 bv{c.box, c.map, c.fib, c.df};
    const DenseOut32 o{c.fn, c.urn, nullptr, nullptr, nullptr};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < w * h; k += gridDim.x * blockDim.x) {
        const int i = x0 + k % w, j = y0 + k / w;
        if (i < 0 || i >= g.nx || j < 0 || j >= g.ny) continue;
        dense_node32<COLL, BC, INCOMP, IBM, false>(c.fp, c.urp, g, c.cp, c.bc, bv, o, i, j);
    }
}

template <int COLL, int BC, bool INCOMP, int IBM>
static cudaError_t launch_batch_kind(const BatchTable& t, int nr, bool box, int box_blocks, cudaStream_t s)
{
    if (box) {
        dense32_box_batch_kernel<COLL, BC, INCOMP, IBM><<<dim3(box_blocks, t.n), 128, 0, s>>>(t);
    } else if (nr == 1) {
        dense32_batch_kernel<COLL, BC, INCOMP, IBM, 1><<<t.off[t.n], 128, 0, s>>>(t);
    } else if (nr == 2) {
        dense32_batch_kernel<COLL, BC, INCOMP, IBM, 2><<<t.off[t.n], 128, 0, s>>>(t);
    } else {
        dense32_batch_kernel<COLL, BC, INCOMP, IBM, 4><<<t.off[t.n], 128, 0, s>>>(t);
    }
    return cudaGetLastError();
}

template <int COLL, int BC, bool INCOMP>
static cudaError_t launch_batch_inc(const BatchTable& t, int ibm, int nr, bool box, int bb, cudaStream_t s)
{
    switch (ibm) {
    case IBM_NONE: return launch_batch_kind<COLL, BC, INCOMP, IBM_NONE>(t, nr, box, bb, s);
    case IBM_DF: return launch_batch_kind<COLL, BC, INCOMP, IBM_DF>(t, nr, box, bb, s);
    case IBM_MDF: return launch_batch_kind<COLL, BC, INCOMP, IBM_MDF>(t, nr, box, bb, s);
    case IBM_DFC: return launch_batch_kind<COLL, BC, INCOMP, IBM_DFC>(t, nr, box, bb, s);
    }
    return cudaErrorInvalidValue;
}

template <int COLL, int BC>
static cudaError_t launch_batch_bc(const BatchTable& t, bool incomp, int ibm, int nr, bool box, int bb, cudaStream_t s)
{
    return incomp ? launch_batch_inc<COLL, BC, true>(t, ibm, nr, box, bb, s)
                  : launch_batch_inc<COLL, BC, false>(t, ibm, nr, box, bb, s);
}

template <int COLL>
static cudaError_t launch_batch_coll(const BatchTable& t, int bc, bool incomp, int ibm, int nr, bool box, int bb,
                                     cudaStream_t s)
{
    switch (bc) {
    case BC_DIRICHLET_NEUMANN: return launch_batch_bc<COLL, BC_DIRICHLET_NEUMANN>(t, incomp, ibm, nr, box, bb, s);
    case BC_OPEN: return launch_batch_bc<COLL, BC_OPEN>(t, incomp, ibm, nr, box, bb, s);
    case BC_SETTLING: return launch_batch_bc<COLL, BC_SETTLING>(t, incomp, ibm, nr, box, bb, s);
    case BC_VELOCITY_INLET: return launch_batch_bc<COLL, BC_VELOCITY_INLET>(t, incomp, ibm, nr, box, bb, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_dense_step_f32_batch(const iblbm_dense32_args* a, int n, void* stream)
{
    if (!a || n < 1 || n > BATCH_MAX) return IBLBM_E_ARG;
    const iblbm_dense32_args& a0 = a[0];
    const bool box = a0.only_box != nullptr;
    int nr = 0;
    if (a0.tile == IBLBM_TILE_NODE) nr = 1;
    else if (a0.tile == IBLBM_TILE_ROWS2) nr = 2;
    else if (a0.tile == IBLBM_TILE_ROWS4) nr = 4;
    else return IBLBM_E_ARG;
    // the parameter block is built on this call's stack and copied into the
    // launch, so concurrent calls from several host threads do not interfere
    BatchTable t;
    t.n = n;
    t.off[0] = 0;
    bool mixed = false;
    for (int b = 0; b < n; ++b) {
        const iblbm_dense32_args& x = a[b];
        if (x.c.collision != a0.c.collision || x.c.bc != a0.c.bc || x.c.incompressible != a0.c.incompressible)
            mixed = true;
        if (x.ibm != a0.ibm || (x.only_box != nullptr) != box || (box && x.skip_box) || x.tile != a0.tile)
            return IBLBM_E_ARG;
        if (x.c.collision < COLL_BGK || x.c.collision > COLL_CMMRT || x.c.bc < 0 || x.c.bc > 3)
            return IBLBM_E_ARG;
        if (x.ro_out || x.U_out || x.fstar_out) return IBLBM_E_ARG;
        if (!x.fpost_prev || !x.fpost_next || x.g.nx < 4 || x.g.ny < 4 || x.g.pitch < x.g.nx) return IBLBM_E_ARG;
        if (9LL * x.g.qstride >= (1LL << 31)) return IBLBM_E_CAPACITY;  // 32-bit pull offsets
        if ((x.c.bc == BC_OPEN || x.c.bc == BC_VELOCITY_INLET) && (!x.uring_prev || !x.uring_next))
            return IBLBM_E_ARG;
        if (x.ibm != IBM_NONE && (!x.band.box || !x.band.map)) return IBLBM_E_ARG;
        if ((x.ibm == IBM_DF || x.ibm == IBM_MDF) && !x.band.fib) return IBLBM_E_ARG;
        if (x.ibm == IBM_DFC && !x.band.df) return IBLBM_E_ARG;
        BatchCase& c = t.c[b];
        c.nx = x.g.nx;
        c.ny = x.g.ny;
        c.pitch = x.g.pitch;
        c.qstride = x.g.qstride;
        c.bx = (x.g.nx + 127) / 128;
        c.kind = x.c.collision * 8 + x.c.bc * 2 + (x.c.incompressible ? 1 : 0);
        c.fp = x.fpost_prev;
        c.fn = x.fpost_next;
        c.urp = x.uring_prev;
        c.urn = x.uring_next;
        c.box = x.band.box;
        c.map = x.band.map;
        c.fib = x.band.fib;
        c.df = x.band.df;
        c.skip_box = x.skip_box;
        c.only_box = x.only_box;
        make_params32(x.c, c.cp, c.bc);
        const long long blocks = (long long)c.bx * ((x.g.ny + nr - 1) / nr);
        if ((long long)t.off[b] + blocks > (1LL << 30)) return IBLBM_E_CAPACITY;
        t.off[b + 1] = t.off[b] + (int)blocks;
    }
    const int bb = a0.box_blocks > 0 ? a0.box_blocks : 16;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (mixed) {
        // cases of several kinds: only bulk passes without a band
        if (box || a0.ibm != IBM_NONE) return IBLBM_E_ARG;
        if (nr == 1) dense32_batch_mixed_kernel<1><<<t.off[n], 128, 0, s>>>(t);
        else if (nr == 2) dense32_batch_mixed_kernel<2><<<t.off[n], 128, 0, s>>>(t);
        else dense32_batch_mixed_kernel<4><<<t.off[n], 128, 0, s>>>(t);
        e = cudaGetLastError();
        return e == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
    }
    switch (a0.c.collision) {
    case COLL_BGK: e = launch_batch_coll<COLL_BGK>(t, a0.c.bc, a0.c.incompressible != 0, a0.ibm, nr, box, bb, s); break;
    case COLL_TRT: e = launch_batch_coll<COLL_TRT>(t, a0.c.bc, a0.c.incompressible != 0, a0.ibm, nr, box, bb, s); break;
    case COLL_CMMRT:
        e = launch_batch_coll<COLL_CMMRT>(t, a0.c.bc, a0.c.incompressible != 0, a0.ibm, nr, box, bb, s);
        break;
    default: return IBLBM_E_ARG;
    }
    return e == cudaSuccess ? IBLBM_OK : (e == cudaErrorInvalidValue ? IBLBM_E_ARG : IBLBM_E_LAUNCH);
}
