// batch_f64.cu — batched FP64 collide-stream pass over many independent cases.
//
// The plain form (the reference's arithmetic, compiled with -fmad=false) of
// the batched pass in batch_f32.cu: many cases of one kind (collision,
// closure, compressibility, band method) advance in one launch.  The per-case
// geometry, pointers and parameters travel in the kernel's parameter block;
// CTA b finds its case by binary search over the cases' block offsets and
// runs the FP64 node pass (dense_node, one node per thread, the same device
// function as the single-case kernel) on one 128-node row segment of that
// case's lattice.  Each case's results are therefore bit-identical to its
// single-case step.
#include "common.cuh"
#include "dense_node.cuh"

namespace iblbm {

void make_params(const iblbm_case& c, CollParams& cp, BcParams& bc);

constexpr int BATCH64_MAX = 72;

struct BatchCase64 {
    int nx, ny, pitch, bx;   // bx: 128-node column blocks
    long long qstride;
    const double* fp;
    double* fn;
    const double* urp;
    double* urn;
    iblbm_band_view band;
    const int* skip_box;
    const int* only_box;
    CollParams cp;
    BcParams bc;
};

struct BatchTable64 {
    int n;
    int off[BATCH64_MAX + 1];
    BatchCase64 c[BATCH64_MAX];
};
// a __grid_constant__ parameter block holds at most 32764 bytes
static_assert(sizeof(BatchTable64) <= 32764, "batched FP64 parameter block too large");

__device__ __forceinline__ int batch64_case(const BatchTable64& t, int blk)
{
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.off[mid] <= blk) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int COLL, int BC, bool INCOMP, int IBM>
__global__ void __launch_bounds__(128) dense64_batch_kernel(const __grid_constant__ BatchTable64 t)
{
    const int ci = batch64_case(t, blockIdx.x);
    const BatchCase64& c = t.c[ci];
    const int local = blockIdx.x - t.off[ci];
    const int i = (local % c.bx) * 128 + threadIdx.x;
    const int j = local / c.bx;
    if (i >= c.nx) return;
    if (c.skip_box) {
        const int x0 = __ldg(c.skip_box + 0), y0 = __ldg(c.skip_box + 1);
        const int w = __ldg(c.skip_box + 2), h = __ldg(c.skip_box + 3);
        if (i >= x0 && i < x0 + w && j >= y0 && j < y0 + h) return;
    }
    const Geom g{c.nx, c.ny, c.pitch, c.qstride};
    const DenseOut o{c.fn, c.urn, nullptr, nullptr, nullptr};
    dense_node<COLL, BC, INCOMP, IBM, false>(c.fp, c.urp, g, c.cp, c.bc, c.band, o, i, j);
}

// Box passes of a batch: blockIdx.y is the case, grid-stride over its box.
template <int COLL, int BC, bool INCOMP, int IBM>
__global__ void __launch_bounds__(128) dense64_box_batch_kernel(const __grid_constant__ BatchTable64 t)
{
    const BatchCase64& c = t.c[blockIdx.y];
    const Geom g{c.nx, c.ny, c.pitch, c.qstride};
    const int x0 = __ldg(c.only_box + 0), y0 = __ldg(c.only_box + 1);
    const int w = __ldg(c.only_box + 2), h = __ldg(c.only_box + 3);
    const DenseOut o{c.fn, c.urn, nullptr, nullptr, nullptr};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < w * h; k += gridDim.x * blockDim.x) {
        const int i = x0 + k % w, j = y0 + k / w;
        if (i < 0 || i >= g.nx || j < 0 || j >= g.ny) continue;
        dense_node<COLL, BC, INCOMP, IBM, false>(c.fp, c.urp, g, c.cp, c.bc, c.band, o, i, j);
    }
}

template <int COLL, int BC, bool INCOMP, int IBM>
static cudaError_t launch64_kind(const BatchTable64& t, bool box, int box_blocks, cudaStream_t s)
{
    if (box) dense64_box_batch_kernel<COLL, BC, INCOMP, IBM><<<dim3(box_blocks, t.n), 128, 0, s>>>(t);
    else dense64_batch_kernel<COLL, BC, INCOMP, IBM><<<t.off[t.n], 128, 0, s>>>(t);
    return cudaGetLastError();
}

template <int COLL, int BC, bool INCOMP>
static cudaError_t launch64_inc(const BatchTable64& t, int ibm, bool box, int bb, cudaStream_t s)
{
    switch (ibm) {
    case IBM_NONE: return launch64_kind<COLL, BC, INCOMP, IBM_NONE>(t, box, bb, s);
    case IBM_DF: return launch64_kind<COLL, BC, INCOMP, IBM_DF>(t, box, bb, s);
    case IBM_MDF: return launch64_kind<COLL, BC, INCOMP, IBM_MDF>(t, box, bb, s);
    case IBM_DFC: return launch64_kind<COLL, BC, INCOMP, IBM_DFC>(t, box, bb, s);
    }
    return cudaErrorInvalidValue;
}

template <int COLL, int BC>
static cudaError_t launch64_bc(const BatchTable64& t, bool incomp, int ibm, bool box, int bb, cudaStream_t s)
{
    return incomp ? launch64_inc<COLL, BC, true>(t, ibm, box, bb, s) : launch64_inc<COLL, BC, false>(t, ibm, box, bb, s);
}

template <int COLL>
static cudaError_t launch64_coll(const BatchTable64& t, int bc, bool incomp, int ibm, bool box, int bb, cudaStream_t s)
{
    switch (bc) {
    case BC_DIRICHLET_NEUMANN: return launch64_bc<COLL, BC_DIRICHLET_NEUMANN>(t, incomp, ibm, box, bb, s);
    case BC_OPEN: return launch64_bc<COLL, BC_OPEN>(t, incomp, ibm, box, bb, s);
    case BC_SETTLING: return launch64_bc<COLL, BC_SETTLING>(t, incomp, ibm, box, bb, s);
    case BC_VELOCITY_INLET: return launch64_bc<COLL, BC_VELOCITY_INLET>(t, incomp, ibm, box, bb, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_dense_step_f64_batch(const iblbm_dense_args* a, int n, void* stream)
{
    if (!a || n < 1 || n > BATCH64_MAX) return IBLBM_E_ARG;
    const iblbm_dense_args& a0 = a[0];
    const bool box = a0.only_box != nullptr;
    BatchTable64 t;  // built per call: concurrent host callers do not interfere
    t.n = n;
    t.off[0] = 0;
    for (int b = 0; b < n; ++b) {
        const iblbm_dense_args& x = a[b];
        if (x.c.collision != a0.c.collision || x.c.bc != a0.c.bc || x.c.incompressible != a0.c.incompressible ||
            x.ibm != a0.ibm || (x.only_box != nullptr) != box || (box && x.skip_box))
            return IBLBM_E_ARG;
        if (x.c.collision < COLL_BGK || x.c.collision > COLL_CMMRT || x.c.bc < 0 || x.c.bc > 3) return IBLBM_E_ARG;
        if (x.ro_out || x.U_out || x.fstar_out) return IBLBM_E_ARG;
        if (!x.fpost_prev || !x.fpost_next || x.g.nx < 4 || x.g.ny < 4 || x.g.pitch < x.g.nx) return IBLBM_E_ARG;
        if ((x.c.bc == BC_OPEN || x.c.bc == BC_VELOCITY_INLET) && (!x.uring_prev || !x.uring_next))
            return IBLBM_E_ARG;
        if (x.ibm != IBM_NONE && (!x.band.box || !x.band.map)) return IBLBM_E_ARG;
        if ((x.ibm == IBM_DF || x.ibm == IBM_MDF) && !x.band.fib) return IBLBM_E_ARG;
        if (x.ibm == IBM_DFC && !x.band.df) return IBLBM_E_ARG;
        BatchCase64& c = t.c[b];
        c.nx = x.g.nx;
        c.ny = x.g.ny;
        c.pitch = x.g.pitch;
        c.qstride = x.g.qstride;
        c.bx = (x.g.nx + 127) / 128;
        c.fp = x.fpost_prev;
        c.fn = x.fpost_next;
        c.urp = x.uring_prev;
        c.urn = x.uring_next;
        c.band = x.band;
        c.skip_box = x.skip_box;
        c.only_box = x.only_box;
        make_params(x.c, c.cp, c.bc);
        const long long blocks = (long long)c.bx * x.g.ny;
        if ((long long)t.off[b] + blocks > (1LL << 30)) return IBLBM_E_CAPACITY;
        t.off[b + 1] = t.off[b] + (int)blocks;
    }
    const int bb = a0.box_blocks > 0 ? a0.box_blocks : 16;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    const bool inc = a0.c.incompressible != 0;
    switch (a0.c.collision) {
    case COLL_BGK: e = launch64_coll<COLL_BGK>(t, a0.c.bc, inc, a0.ibm, box, bb, s); break;
    case COLL_TRT: e = launch64_coll<COLL_TRT>(t, a0.c.bc, inc, a0.ibm, box, bb, s); break;
    case COLL_CMMRT: e = launch64_coll<COLL_CMMRT>(t, a0.c.bc, inc, a0.ibm, box, bb, s); break;
    default: return IBLBM_E_ARG;
    }
    return e == cudaSuccess ? IBLBM_OK : (e == cudaErrorInvalidValue ? IBLBM_E_ARG : IBLBM_E_LAUNCH);
}
