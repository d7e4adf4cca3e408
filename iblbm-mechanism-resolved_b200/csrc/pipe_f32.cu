// pipe_f32.cu — pipelined FP32 collide-stream pass (shared-memory staging by
// bulk copies).  Split from dense_f32.cu so the units compile in parallel.
#include <cstdint>
#include "shifted.cuh"
#include "tma.cuh"

namespace iblbm {

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
    case BC_TG:
        dense_node32<COLL, BC_TG, INCOMP, IBM, false>(a.fpost_prev, a.uring_prev, g, cp, bc, bv, o, i, j);
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
    const long long wait_limit = a.wait_limit > 0 ? a.wait_limit : PIPE_WAIT_LIMIT;
    if (warp == ROWS) {
        // producer (test_skip_copy: issues nothing, so every consumer wait runs out)
        if (a.test_skip_copy) return;
        int k = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
            const int s = k % STAGES;
            if (k >= STAGES && !mbar_wait_bounded(&empty[s], ((k / STAGES) & 1) ^ 1, wait_limit)) {
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
        if (!mbar_wait_bounded(&full[s], (k / STAGES) & 1, wait_limit)) {
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

template <int COLL, bool RING, bool INCOMP>
static cudaError_t pipe_ibm(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
#define IBLBM_PIPE(IBMV)                                                                                   \
    return a.tile == IBLBM_TILE_PIPE_8x2 ? launch_pipe<COLL, RING, INCOMP, IBMV, 8, 2, 2>(a, cp, bc, s) \
                                         : launch_pipe<COLL, RING, INCOMP, IBMV, 4, 2, 5>(a, cp, bc, s)
    switch (a.ibm) {
    case IBM_NONE: IBLBM_PIPE(IBM_NONE);
    case IBM_DF: IBLBM_PIPE(IBM_DF);
    case IBM_MDF: IBLBM_PIPE(IBM_MDF);
    case IBM_DFC: IBLBM_PIPE(IBM_DFC);
    }
#undef IBLBM_PIPE
    return cudaErrorInvalidValue;
}

template <int COLL, bool RING>
static cudaError_t pipe_inc(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    return a.c.incompressible ? pipe_ibm<COLL, RING, true>(a, cp, bc, s) : pipe_ibm<COLL, RING, false>(a, cp, bc, s);
}

template <int COLL>
static cudaError_t pipe_ring(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    const bool ring = a.c.bc == BC_OPEN || a.c.bc == BC_VELOCITY_INLET;
    return ring ? pipe_inc<COLL, true>(a, cp, bc, s) : pipe_inc<COLL, false>(a, cp, bc, s);
}

// Launch the pipelined whole-lattice / bulk pass (tile IBLBM_TILE_PIPE_*).
cudaError_t launch_pipe32(const iblbm_dense32_args& a, const CollParams32& cp, const BcParams32& bc, cudaStream_t s)
{
    switch (a.c.collision) {
    case COLL_BGK: return pipe_ring<COLL_BGK>(a, cp, bc, s);
    case COLL_TRT: return pipe_ring<COLL_TRT>(a, cp, bc, s);
    case COLL_CMMRT: return pipe_ring<COLL_CMMRT>(a, cp, bc, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace iblbm
