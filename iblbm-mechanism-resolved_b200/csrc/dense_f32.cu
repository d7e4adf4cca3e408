// dense_f32.cu — fused timestep in the FP32 shifted-population form.
//
// Same schedule as dense_f64.cu (pull-stream, closure, band correction,
// moments, velocity correction, equilibrium, collision, store) on deviations
// g = f - w held in FP32: 72 bytes per lattice update.  Compiled with the
// default multiply-add contraction.
#include <cstdint>
#include "shifted.cuh"
#include "tma.cuh"

namespace iblbm {

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
    float f[NR][9];
#pragma unroll
    for (int n = 0; n < NR; ++n)
        if (j0 + n < g.ny) pull(a.fpost_prev, g, i, j0 + n, f[n]);
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

// ---------------------------------------------------------------------------
// Pipelined pass: persistent CTAs, one producer warp staging each tile's
// population rows into shared memory with bulk copies (cp.async.bulk, completing
// on an mbarrier), ROWS consumer warps computing from shared memory and storing
// straight to global memory.  A tile is ROWS lattice rows x PIPE_W columns; the
// stage buffer holds, for every population plane q, the rows y0 + r - ey(q)
// (r < ROWS) over columns x0 - 4 .. x0 + PIPE_W + 3, so every pull source of
// the tile's interior nodes is on chip.  STAGES buffers rotate: while the
// consumers work on one tile the copies of the next STAGES - 1 are in flight.
// Edge nodes of the lattice take the per-node path (closures read global
// memory); nodes in the skip box are left to the box pass.
// ---------------------------------------------------------------------------
constexpr int PIPE_W = 128;
constexpr int PIPE_SW = PIPE_W + 8;
constexpr long long PIPE_WAIT_LIMIT = 1LL << 24;
constexpr int PIPE_TIMEOUT = 1;  // status code: a pipeline wait ran out

template <int ROWS, int STAGES>
constexpr size_t pipe_smem_bytes() { return sizeof(float) * (size_t)STAGES * 9 * ROWS * PIPE_SW; }

template <int COLL, bool INCOMP, int IBM>
__device__ __forceinline__ void node_generic32(const iblbm_dense32_args& a, const Geom& g, const CollParams32& cp,
                                               const BcParams32& bc, const BandView32& bv, const DenseOut32& o,
                                               int i, int j)
{
    switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN:
        dense_node32<COLL, BC_DIRICHLET_NEUMANN, INCOMP, IBM, false>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
        break;
    case BC_OPEN:
        dense_node32<COLL, BC_OPEN, INCOMP, IBM, false>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
        break;
    case BC_SETTLING:
        dense_node32<COLL, BC_SETTLING, INCOMP, IBM, false>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
        break;
    default:
        dense_node32<COLL, BC_VELOCITY_INLET, INCOMP, IBM, false>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i,
                                                                   j);
        break;
    }
}

template <int COLL, bool RING, bool INCOMP, int IBM, int ROWS, int STAGES, int MINB>
__global__ void __launch_bounds__(32 * (ROWS + 1), MINB) dense32_pipe_kernel(const iblbm_dense32_args a, CollParams32 cp,
                                                                     BcParams32 bc)
{
    extern __shared__ __align__(128) float psm[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntx = (g.nx + PIPE_W - 1) / PIPE_W, nty = (g.ny + ROWS - 1) / ROWS;
    const int ntiles = ntx * nty;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], ROWS);
        }
    }
    __syncthreads();
    int sx0 = 0, sy0 = 0, sx1 = -1, sy1 = -1;
    if (a.skip_box) {
        sx0 = __ldg(a.skip_box + 0);
        sy0 = __ldg(a.skip_box + 1);
        sx1 = sx0 + __ldg(a.skip_box + 2) - 1;
        sy1 = sy0 + __ldg(a.skip_box + 3) - 1;
    }
    constexpr int STAGE_F = 9 * ROWS * PIPE_SW;
    if (warp == ROWS) {
        // producer
        int k = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
            const int s = k % STAGES;
            if (k >= STAGES && !mbar_wait_bounded(&empty[s], ((k / STAGES) & 1) ^ 1, PIPE_WAIT_LIMIT)) {
                if (lane == 0 && a.status) atomicExch(a.status, PIPE_TIMEOUT);
                break;
            }
            const int x0 = (t % ntx) * PIPE_W, y0 = (t / ntx) * ROWS;
            const int c0 = max(x0 - 4, 0), c1 = min(x0 + PIPE_W + 4, g.pitch);
            const uint32_t row_bytes = (uint32_t)(c1 - c0) * 4u;
            if (lane == 0) {
                uint32_t total = 0;
                for (int c = 0; c < 9 * ROWS; ++c) {
                    const int row = y0 + c % ROWS - ey_(c / ROWS);
                    if (row >= 0 && row < g.ny) total += row_bytes;
                }
                mbar_expect(&full[s], total);
            }
            __syncwarp();
            float* st = psm + (size_t)s * STAGE_F;
            for (int c = lane; c < 9 * ROWS; c += 32) {
                const int q = c / ROWS, r = c % ROWS;
                const int row = y0 + r - ey_(q);
                if (row < 0 || row >= g.ny) continue;
                bulk_copy(st + (q * ROWS + r) * PIPE_SW + (c0 - (x0 - 4)),
                          a.fpost_prev + q * g.qstride + (long long)row * g.pitch + c0, row_bytes, &full[s]);
            }
        }
        return;
    }
    // consumers: warp r computes row y0 + r of each tile
    const BandView32 bv{a.band.box, a.band.map, a.band.fib, a.band.df};
    const DenseOut32 o{a.fpost_next, a.uring_next, nullptr, nullptr, nullptr};
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        const int s = k % STAGES;
        if (!mbar_wait_bounded(&full[s], (k / STAGES) & 1, PIPE_WAIT_LIMIT)) {
            if (lane == 0 && a.status) atomicExch(a.status, PIPE_TIMEOUT);
            break;
        }
        const int x0 = (t % ntx) * PIPE_W, y0 = (t / ntx) * ROWS;
        const int j = y0 + warp;
        const float* st = psm + (size_t)s * STAGE_F + warp * PIPE_SW;
        if (j < g.ny) {
            const bool row_in = j >= 1 && j <= g.ny - 2;
            const bool row_skip = j >= sy0 && j <= sy1;
#pragma unroll 1
            for (int ii = 0; ii < PIPE_W / 32; ++ii) {
                const int i = x0 + ii * 32 + lane;
                if (i >= g.nx || (row_skip && i >= sx0 && i <= sx1)) continue;
                if (row_in && i >= 1 && i <= g.nx - 2) {
                    float f[9], out[9];
                    const int c = i - x0 + 4;
#pragma unroll
                    for (int q = 0; q < 9; ++q) f[q] = st[q * ROWS * PIPE_SW + c - ex_(q)];
                    node_core32<COLL, RING, INCOMP, IBM, false>(f, g, cp, bv, o, i, j, out);
                    float* dst = a.fpost_next + (long long)j * g.pitch + i;
#pragma unroll
                    for (int q = 0; q < 9; ++q) dst[q * g.qstride] = out[q];
                } else {
                    node_generic32<COLL, INCOMP, IBM>(a, g, cp, bc, bv, o, i, j);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// Persistent grid of one pipelined instantiation: resident CTAs per SM x SMs,
// at most one CTA per tile.  The first launch of each sets its shared-memory
// limit and reads the occupancy (for the device current at that call).
template <int COLL, bool RING, bool INCOMP, int IBM, int ROWS, int STAGES, int MINB>
static cudaError_t launch_pipe(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    auto K = dense32_pipe_kernel<COLL, RING, INCOMP, IBM, ROWS, STAGES, MINB>;
    constexpr size_t smem = pipe_smem_bytes<ROWS, STAGES>();
    constexpr int threads = 32 * (ROWS + 1);
    static int per_sm = 0, sms = 0;
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int dev = 0, n = 0, occ = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, K, threads, smem)) != cudaSuccess) return e;
        if (occ < 1) return cudaErrorInvalidConfiguration;
        sms = n;
        per_sm = occ;
    }
    const int ntiles = ((a.g.nx + PIPE_W - 1) / PIPE_W) * ((a.g.ny + ROWS - 1) / ROWS);
    const int grid = min(ntiles, per_sm * sms);
    K<<<grid, threads, smem, s>>>(a, cp, bc);
    return cudaGetLastError();
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
    // the pipelined pass dispatches the closures at run time: its instantiations
    // depend on the boundary only through the velocity ring
    constexpr bool RING = has_ring<BC>();
    if (a.tile == IBLBM_TILE_ROWS2 || a.tile == IBLBM_TILE_ROWS4) {
        const int nr = a.tile == IBLBM_TILE_ROWS2 ? 2 : 4;
        dim3 grid((a.g.nx + 127) / 128, (a.g.ny + nr - 1) / nr);
        if (nr == 2) dense32_rows_kernel<COLL, BC, INCOMP, IBM, 2><<<grid, 128, 0, s>>>(a, cp, bc);
        else dense32_rows_kernel<COLL, BC, INCOMP, IBM, 4><<<grid, 128, 0, s>>>(a, cp, bc);
        return cudaGetLastError();
    }
    if (a.tile == IBLBM_TILE_PIPE_8x2) return launch_pipe<COLL, RING, INCOMP, IBM, 8, 2, 2>(a, cp, bc, s);
    return launch_pipe<COLL, RING, INCOMP, IBM, 4, 2, 5>(a, cp, bc, s);
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

template <int COLL, int BC, bool INCOMP, int IBM, int NR>
__global__ void __launch_bounds__(128) dense32_batch_kernel(const __grid_constant__ BatchTable t)
{
    const int ci = batch_case(t, blockIdx.x);
    const BatchCase& c = t.c[ci];
    const int local = blockIdx.x - t.off[ci];
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
    float f[NR][9];
#pragma unroll
    for (int n = 0; n < NR; ++n)
        if (j0 + n < g.ny) pull(c.fp, g, i, j0 + n, f[n]);
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
    static BatchTable t;  // host staging of the parameter block (calls are serialised by the caller)
    t.n = n;
    t.off[0] = 0;
    for (int b = 0; b < n; ++b) {
        const iblbm_dense32_args& x = a[b];
        if (x.c.collision != a0.c.collision || x.c.bc != a0.c.bc || x.c.incompressible != a0.c.incompressible ||
            x.ibm != a0.ibm || (x.only_box != nullptr) != box || (box && x.skip_box) || x.tile != a0.tile)
            return IBLBM_E_ARG;
        if (x.ro_out || x.U_out || x.fstar_out) return IBLBM_E_ARG;
        if (!x.fpost_prev || !x.fpost_next || x.g.nx < 4 || x.g.ny < 4 || x.g.pitch < x.g.nx) return IBLBM_E_ARG;
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
