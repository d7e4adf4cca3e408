// band_kernel.cuh — immersed-boundary marker loop on the band.
//
// The band is the set of lattice nodes under the marker stencils (a few hundred
// to a few thousand nodes).  One CTA of 512 threads owns it for the whole step:
//
//   rebuild (fixed bodies: once; moving bodies: every step)
//     markers -> nearest node ix0 = floor(x/dx + 0.5) and separable weights
//     wx[2a+1], wy[2a+1]; bounding box; band compaction in row-major (= lattice
//     index) order; per-node contribution lists sorted by stencil slot k
//     (di outer, dj inner) then marker l — the order in which numpy's add.at
//     applies the reference's scatter — with each entry's spreading weight
//     (wx*wy)*ds precomputed.
//   every step
//     for fixed bodies the per-step-constant block (slot -> band index, lists,
//     weights, node list, stencil origins) is restored into shared memory from its global cache
//     with one TMA bulk copy (cp.async.bulk + mbarrier) while the marker data
//     loads; then post-streaming populations and moments on the band (the
//     dense kernel's device functions), and DF, MDF (every iteration resident
//     on chip: two barriers per iteration, residual reduced in shared memory,
//     no host round trip; the FP32 form iterates a single body on its markers
//     through a banded marker coupling matrix, one barrier per iteration),
//     coupled multi-particle MDF, or DFC.
//   exclusion box
//     the band's bounding box dilated by one node is written for the next
//     step: markers move less than one node per step, so the next band lies
//     inside it.  The bulk collide-stream kernel of the next step skips that
//     box and runs concurrently with this kernel; a small box kernel updates
//     the box once this kernel has produced the band forces.
//
// Two instantiations: R = double on the FP64 lattice (ibm_f64.cu, compiled
// without multiply-add contraction: every sum runs in the reference's order and
// results are bit-identical to the reference CPU path), and R = float on the
// shifted FP32 lattice (ibm_f32.cu), where the MDF residual norm stays FP64.
//
// The kernel is latency-bound (one CTA, dependent sums in a fixed order): every
// loop over stencil slots or list entries is unrolled so its loads issue
// together and only the sum itself is serial.
#pragma once
#include <climits>
#include <cstdint>
#include <type_traits>
#include "common.cuh"
#include "shifted.cuh"
#include "tma.cuh"
#include "mlp.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int IBM_THREADS = 512;
constexpr int NPT = 4;          // band nodes per thread in the MDF loop
constexpr int MAX_BAND = NPT * IBM_THREADS;  // band capacity limit (2048)
constexpr int MAXP = 8;    // particles per band kernel
constexpr int NWARP = IBM_THREADS / 32;
constexpr long long TMA_WAIT_LIMIT = 1LL << 22;
constexpr int IBM_SMEM_LIMIT = 220 * 1024;
enum IbmStatus : int { ST_OK = 0, ST_BAND_CAPACITY = 1, ST_BOX_CAPACITY = 2, ST_MARKERS = 3, ST_TABLE = 4,
                       ST_EXCL = 5, ST_COPY_TIMEOUT = 6 };

template <int A>
struct Sten {
    static constexpr int SW = 2 * A + 1;
    static constexpr int S = SW * SW;
};

__host__ __device__ inline size_t up16(size_t x) { return (x + 15) & ~size_t(15); }

constexpr int MLP_CHUNK = IBM_THREADS / 4;  // markers per network tile (128)

// Shared memory of the learned warm start, placed after the band layout: two
// activation tiles, the outputs of a tile, the predicted force per marker, and
// the header of the network's parameter block (restored by one bulk copy at
// kernel start).
__host__ __device__ inline size_t mlp_act_bytes(int Lb)
{
    return up16(sizeof(float) * ((size_t)2 * MLP_CHUNK * MLP_LD + 2 * MLP_CHUNK + 4 * (size_t)Lb + MLP_WBUF));
}
// (only the parameter block's header, the feature normalisation and target
// scales, is copied; the layers read their weights from global memory, where
// the 57 KB block stays in L1 / L2)
__host__ __device__ inline size_t mlp_smem_bytes(int Lb) { return mlp_act_bytes(Lb) + sizeof(float) * MLP_HDR; }

// Marker-space MDF of the FP32 form: row l of the marker coupling matrix keeps
// the markers l - MS_D .. l + MS_D (neighbours along the body).
constexpr int MS_D = 8;
constexpr int MS_W = 2 * MS_D + 1;
// The matrix, then per stencil slot W_lk vs(b_k) while it is built, whose room
// the two force buffers of the iterations take over.
__host__ __device__ inline size_t ms_smem_bytes(int Lb, int S)
{
    const size_t build = (size_t)Lb * S, iterate = 4 * ((size_t)Lb + 2 * MS_D);
    return up16(sizeof(float) * ((size_t)Lb * MS_W + (build > iterate ? build : iterate)));
}
// Whether the marker-space loop runs: a ring of at least MS_W markers (so the
// MS_W neighbours of a marker are distinct) whose matrix fits beside the band
// layout (`base` bytes).  Host sizing and kernel use the same test.
__host__ __device__ inline bool ms_fits(size_t base, int Lb, int S)
{
    return Lb >= MS_W && base + ms_smem_bytes(Lb, S) <= (size_t)IBM_SMEM_LIMIT;
}
__device__ __forceinline__ int ms_ring(int m, int Lb) { return m + (m < 0 ? Lb : 0) - (m >= Lb ? Lb : 0); }

// Node-space MDF of one body in the FP64 form, restructured for the shared
// memory of one CTA (same operations in the same order as the plain loop, so
// the same bits).  An iteration is bound by shared-memory traffic: gathers of
// the band velocities and of the marker forces, FP64 words with bank
// conflicts.  Each band node therefore walks its contribution list in
// jagged-diagonal order (list position j of the nodes ranked by list length
// lies contiguously), so a warp's list loads are consecutive words, and the
// residual is one maximum over squared slips.  Shared memory after the band
// layout: staging of the reordered lists, and per rank the node and its list
// length, the jagged-diagonal offsets and a histogram of list lengths.
constexpr int NSF_MAX_MARKERS = IBM_THREADS;  // one thread per marker
__host__ __device__ inline size_t nsf_stage_bytes(int Lb, int S)
{
    return up16(sizeof(int) * (size_t)Lb * S) + up16(sizeof(double) * (size_t)Lb * S);
}
__host__ __device__ inline size_t nsf_smem_bytes(int Lb, int NB, int S)
{
    return nsf_stage_bytes(Lb, S) + up16(sizeof(int) * (2 * (size_t)NB + 3 * ((size_t)S + 2)));
}
// Whether the restructured loop runs: a body of at most NSF_MAX_MARKERS
// markers whose extra room fits beside the band layout (`base` bytes).  Host
// sizing and kernel use the same test.
__host__ __device__ inline bool nsf_fits(size_t base, int Lb, int NB, int S)
{
    return Lb <= NSF_MAX_MARKERS && base + nsf_smem_bytes(Lb, NB, S) <= (size_t)IBM_SMEM_LIMIT;
}
// Barrier `id` over the first n threads of the block (n a multiple of 32).
__device__ __forceinline__ void bar_sync_n(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
inline bool mlp_on(const iblbm_ibm_args&) { return false; }
inline bool ms_on(const iblbm_ibm_args&) { return false; }
inline bool ms_on(const iblbm_ibm32_args& a) { return a.method == IBM_MDF && !a.mdf_coupled; }
inline bool nsf_on(const iblbm_ibm_args& a) { return a.method == IBM_MDF && !a.mdf_coupled; }
inline bool nsf_on(const iblbm_ibm32_args&) { return false; }
inline bool mlp_on(const iblbm_ibm32_args& a)
{
    return a.mlp_mode != 0 && a.method == IBM_MDF && !a.mdf_coupled;
}


// Shared-memory layout.  The "static" block (everything a fixed body keeps
// between steps) is contiguous so that one bulk copy restores it.
struct Layout {
    size_t o_sidx, o_ent, o_cstart, o_nodes, o_part, o_wx, o_wy, o_entw, o_ix0, o_iy0, static_bytes;
    size_t o_dvx, o_dvy, o_R, o_Lux, o_Luy, o_Lfx, o_Lfy, o_bro, o_bwx, o_bwy, o_wred, o_ired, total;
};

template <typename R>
__host__ __device__ inline Layout make_layout(int Lb, int NB, int S)
{
    Layout L;
    size_t o = 0;
    L.o_sidx = o; o = up16(o + sizeof(int) * (size_t)Lb * S);
    L.o_ent = o; o = up16(o + sizeof(int) * (size_t)Lb * S);
    L.o_cstart = o; o = up16(o + sizeof(int) * ((size_t)NB + 1));
    L.o_nodes = o; o = up16(o + sizeof(int) * (size_t)NB);
    L.o_part = o; o = up16(o + sizeof(int) * (size_t)Lb);
    L.o_wx = o; o = up16(o + sizeof(R) * (size_t)Lb * 5);
    L.o_wy = o; o = up16(o + sizeof(R) * (size_t)Lb * 5);
    L.o_entw = o; o = up16(o + sizeof(R) * (size_t)Lb * S);
    L.o_ix0 = o; o = up16(o + sizeof(int) * (size_t)Lb);
    L.o_iy0 = o; o = up16(o + sizeof(int) * (size_t)Lb);
    L.static_bytes = o;
    L.o_dvx = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_dvy = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_R = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_Lux = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_Luy = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_Lfx = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_Lfy = o; o = up16(o + sizeof(R) * (size_t)Lb);
    L.o_bro = o; o = up16(o + sizeof(R) * (size_t)NB);
    L.o_bwx = o; o = up16(o + sizeof(R) * (size_t)NB);
    L.o_bwy = o; o = up16(o + sizeof(R) * (size_t)NB);
    L.o_wred = o; o = up16(o + sizeof(double) * 2 * MAXP * NWARP);
    L.o_ired = o; o = up16(o + sizeof(int) * 64);
    L.total = o;
    return L;
}

template <typename R>
struct Sm {
    int *sidx, *ent, *cstart, *nodes, *part, *ix0, *iy0, *ired;
    R *wx, *wy, *entw, *dvx, *dvy, *R_, *Lux, *Luy, *Lfx, *Lfy, *bro, *bwx, *bwy;
    double* wred;  // per-warp residual maxima (FP64 in both forms)
};

// The per-step-constant block (lists, stencil weights and origins) at sbase,
// the rest at dbase, shifted down by `shift` bytes (the static block's size
// when it lives elsewhere; every dynamic offset is at least that).
template <typename R>
__device__ inline Sm<R> carve2(char* sbase, char* dbase, const Layout& L, size_t shift)
{
    Sm<R> s;
    s.sidx = reinterpret_cast<int*>(sbase + L.o_sidx);
    s.ent = reinterpret_cast<int*>(sbase + L.o_ent);
    s.cstart = reinterpret_cast<int*>(sbase + L.o_cstart);
    s.nodes = reinterpret_cast<int*>(sbase + L.o_nodes);
    s.part = reinterpret_cast<int*>(sbase + L.o_part);
    s.wx = reinterpret_cast<R*>(sbase + L.o_wx);
    s.wy = reinterpret_cast<R*>(sbase + L.o_wy);
    s.entw = reinterpret_cast<R*>(sbase + L.o_entw);
    s.ix0 = reinterpret_cast<int*>(sbase + L.o_ix0);
    s.iy0 = reinterpret_cast<int*>(sbase + L.o_iy0);
    s.dvx = reinterpret_cast<R*>(dbase + (L.o_dvx - shift));
    s.dvy = reinterpret_cast<R*>(dbase + (L.o_dvy - shift));
    s.R_ = reinterpret_cast<R*>(dbase + (L.o_R - shift));
    s.Lux = reinterpret_cast<R*>(dbase + (L.o_Lux - shift));
    s.Luy = reinterpret_cast<R*>(dbase + (L.o_Luy - shift));
    s.Lfx = reinterpret_cast<R*>(dbase + (L.o_Lfx - shift));
    s.Lfy = reinterpret_cast<R*>(dbase + (L.o_Lfy - shift));
    s.bro = reinterpret_cast<R*>(dbase + (L.o_bro - shift));
    s.bwx = reinterpret_cast<R*>(dbase + (L.o_bwx - shift));
    s.bwy = reinterpret_cast<R*>(dbase + (L.o_bwy - shift));
    s.wred = reinterpret_cast<double*>(dbase + (L.o_wred - shift));
    s.ired = reinterpret_cast<int*>(dbase + (L.o_ired - shift));
    return s;
}

template <typename R>
__device__ inline Sm<R> carve(char* base, const Layout& L)
{
    return carve2<R>(base, base, L, 0);
}

__device__ __forceinline__ double nanmax(double a, double b) { return (b > a || b != b) ? b : a; }

// Warp maximum of 64-bit patterns of non-negative doubles or NaNs: for those
// the unsigned order of the patterns is the numeric order, with every NaN above
// every number (as nanmax keeps a NaN).
__device__ __forceinline__ unsigned long long warp_max_bits(unsigned long long v)
{
    const unsigned hi = (unsigned)(v >> 32);
    const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? (unsigned)v : 0u);
    return ((unsigned long long)mh << 32) | ml;
}

__device__ __forceinline__ double warp_nanmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide exclusive scan of one int per thread; returns the prefix, writes the total.
__device__ inline int block_exscan(int v, int* ired, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += u;
    }
    __syncthreads();
    if (lane == 31) ired[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int y = lane < NWARP ? ired[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += u;
        }
        if (lane < NWARP) ired[32 + lane] = y;
    }
    __syncthreads();
    const int base = wid > 0 ? ired[32 + wid - 1] : 0;
    *total = ired[32 + NWARP - 1];
    __syncthreads();
    return base + x - v;
}

// e . u in the precision R (the FP64 instance is e_dot)
template <typename R>
__device__ __forceinline__ R edot_r(int q, R u0, R u1)
{
    const R a = (R)ex_(q) * u0;
    const R b = (R)ey_(q) * u1;
    return a + b;
}

// Post-streaming populations and moments of the band nodes; two nodes per pass
// so their global loads are in flight together.  The FP64 form keeps f*, the
// shifted form g* = f* - w (the DFC correction is the same in both, since the
// bounce-back deviation pairs equal weights).
template <bool SHIFTED, int BC, class ARGS, class BCP, typename R>
__device__ void band_moments(const ARGS& a, const Geom& g, const BCP& bc, int nb, Sm<R>& sh, R* bfs)
{
    const bool incomp = a.c.incompressible != 0;
    for (int b0 = threadIdx.x; b0 < nb; b0 += 2 * IBM_THREADS) {
        const int b1 = b0 + IBM_THREADS;
        const bool two = b1 < nb;
        const int n0 = sh.nodes[b0], n1 = sh.nodes[two ? b1 : b0];
        const int j0 = n0 / g.nx, i0 = n0 - j0 * g.nx, j1 = n1 / g.nx, i1 = n1 - j1 * g.nx;
        R f0[9], f1[9], r0, x0, y0, r1, x1, y1;
        if constexpr (SHIFTED) {
            gstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i0, j0, f0);
            gstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i1, j1, f1);
            float d0, d1;
            macro_g(f0, incomp, d0, r0, x0, y0);
            macro_g(f1, incomp, d1, r1, x1, y1);
        } else {
            fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i0, j0, f0);
            fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i1, j1, f1);
            macro_seq(f0, incomp, r0, x0, y0);
            macro_seq(f1, incomp, r1, x1, y1);
        }
        sh.bro[b0] = r0; sh.bwx[b0] = x0; sh.bwy[b0] = y0;
        if (bfs) {
#pragma unroll
            for (int q = 0; q < 9; ++q) bfs[9 * (size_t)b0 + q] = f0[q];
        }
        if (two) {
            sh.bro[b1] = r1; sh.bwx[b1] = x1; sh.bwy[b1] = y1;
            if (bfs) {
#pragma unroll
                for (int q = 0; q < 9; ++q) bfs[9 * (size_t)b1 + q] = f1[q];
            }
        }
    }
}

// Band moments of a reference-shaped call: density and velocity, or the
// post-streaming populations, read from the caller's fields.
template <class ARGS, typename R>
__device__ void field_moments(const ARGS& a, int nb, Sm<R>& sh, R* bfs)
{
    const int s = a.field_ustride > 0 ? a.field_ustride : 1;
    for (int b = threadIdx.x; b < nb; b += IBM_THREADS) {
        const long long n = sh.nodes[b];
        if (bfs) {
#pragma unroll
            for (int q = 0; q < 9; ++q) bfs[9 * (size_t)b + q] = a.field_fstar[9 * n + q];
        } else {
            sh.bro[b] = a.field_ro[n];
            sh.bwx[b] = a.field_ux[n * s];
            sh.bwy[b] = a.field_uy[n * s];
        }
    }
}

template <int A, typename R>
__device__ __forceinline__ R wgt(const Sm<R>& sh, int l, int k)
{
    constexpr int SW = Sten<A>::SW;
    return sh.wx[l * 5 + k / SW] * sh.wy[l * 5 + k % SW];
}

// Interpolate two band fields at marker l: (sum_k u[b_k] w_k, sum_k v[b_k] w_k)
// in slot order, loads issued together.
template <int A, typename R>
__device__ __forceinline__ void interp2(const Sm<R>& sh, const R* u, const R* v, int l, R& su, R& sv)
{
    constexpr int S = Sten<A>::S;
    int bk[S];
    R wk[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        bk[k] = sh.sidx[l * S + k];
        wk[k] = wgt<A>(sh, l, k);
    }
    R x = 0, y = 0;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        x += u[bk[k]] * wk[k];
        y += v[bk[k]] * wk[k];
    }
    su = x;
    sv = y;
}

// Sequential sum over list entries [u0, u1) of g[l] * w (entries' own weights),
// unrolled by 4 so the loads of four entries are in flight together.
template <typename R>
__device__ __forceinline__ void spread2(const Sm<R>& sh, const R* gx, const R* gy, int u0, int u1, R& ax, R& ay)
{
    R x = 0, y = 0;
    int u = u0;
    for (; u + 4 <= u1; u += 4) {
        const int e0 = sh.ent[u], e1 = sh.ent[u + 1], e2 = sh.ent[u + 2], e3 = sh.ent[u + 3];
        const R w0 = sh.entw[u], w1 = sh.entw[u + 1], w2 = sh.entw[u + 2], w3 = sh.entw[u + 3];
        const int l0 = e0 >> 5, l1 = e1 >> 5, l2 = e2 >> 5, l3 = e3 >> 5;
        const R p0 = gx[l0] * w0, p1 = gx[l1] * w1, p2 = gx[l2] * w2, p3 = gx[l3] * w3;
        const R q0 = gy[l0] * w0, q1 = gy[l1] * w1, q2 = gy[l2] * w2, q3 = gy[l3] * w3;
        x += p0; x += p1; x += p2; x += p3;
        y += q0; y += q1; y += q2; y += q3;
    }
    for (; u < u1; ++u) {
        const int l = sh.ent[u] >> 5;
        const R w = sh.entw[u];
        x += gx[l] * w;
        y += gy[l] * w;
    }
    ax = x;
    ay = y;
}

template <bool SHIFTED>
using BcOf = typename std::conditional<SHIFTED, BcParams32, BcParams>::type;

// The band step of one case, run by one CTA of IBM_THREADS threads.  With GS
// the per-step-constant block (contribution lists, stencil weights, origins)
// stays in global memory (list_cache, L2-resident) instead of shared memory:
// the form for bodies whose lists do not fit on chip.
template <class ARGS, typename R, bool SHIFTED, int A, int METHOD, bool COUPLED, bool GS = false>
__device__ __forceinline__ void ibm_step_body(const ARGS& a, const BcOf<SHIFTED>& bc)
{
    constexpr int SW = Sten<A>::SW, S = Sten<A>::S;
    extern __shared__ __align__(16) char smem_raw[];
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int P = a.n_particles, Lb = a.lb_total, NB = a.band_capacity;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const Layout Lay = make_layout<R>(Lb, NB, S);
    const size_t dyn_end = Lay.total - (GS ? Lay.static_bytes : 0);  // shared bytes of the layout
    Sm<R> sh;
    if constexpr (GS) sh = carve2<R>(reinterpret_cast<char*>(a.list_cache), smem_raw, Lay, Lay.static_bytes);
    else sh = carve<R>(smem_raw, Lay);
    __shared__ int s_nb, s_status, s_box[4], s_step, s_cur;
    __shared__ __align__(8) uint64_t s_bar, s_wbar;
    const bool rebuild = a.rebuild || a.xt_table;
    const long long wait_limit = a.wait_limit > 0 ? a.wait_limit : TMA_WAIT_LIMIT;
    // an early return first waits (bounded) for the network copy in flight
    auto drain_weights = [&]() {
        if constexpr (SHIFTED && METHOD == IBM_MDF && !COUPLED) {
            if (a.mlp_mode & 2) mbar_wait_bounded(&s_wbar, 0, wait_limit);
        }
    };
    if constexpr (SHIFTED && METHOD == IBM_MDF && !COUPLED) {
        // the warm start's normalisation header: one bulk copy into shared memory, waited for
        // just before its first use
        if (tid == 0 && (a.mlp_mode & 2)) {
            mbar_init(&s_wbar);
            mbar_expect(&s_wbar, (uint32_t)(sizeof(float) * MLP_HDR));
            bulk_copy(smem_raw + dyn_end + mlp_act_bytes(Lb), a.mlp_params, (uint32_t)(sizeof(float) * MLP_HDR),
                      &s_wbar);
        }
    }
    if (tid == 0) {
        s_status = ST_OK;
        s_step = a.step_counter ? *a.step_counter : 0;
        if (a.xt_table && (s_step < 0 || s_step >= a.xt_len)) s_status = ST_TABLE;
        if (!rebuild && s_status == ST_OK) {
            if constexpr (!GS) {
                // restore the per-step-constant block of a fixed body in one bulk copy
                mbar_init(&s_bar);
                const uint32_t bytes = (uint32_t)Lay.static_bytes;
                mbar_expect(&s_bar, bytes);
                const char* src = reinterpret_cast<const char*>(a.list_cache);
                // (test_skip_copy: the wait below runs out with nothing in flight)
                for (uint32_t off = 0; off < (a.test_skip_copy ? 0u : bytes); off += 65536u) {
                    const uint32_t chunk = min(65536u, bytes - off);
                    bulk_copy(smem_raw + off, src + off, chunk, &s_bar);
                }
            }
            s_nb = *a.band_count;
            s_box[0] = a.box[0];
            s_box[1] = a.box[1];
            s_box[2] = a.box[0] + a.box[2] - 1;
            s_box[3] = a.box[1] + a.box[3] - 1;
        }
    }
    __syncthreads();
    if (s_status != ST_OK) {
        if (tid == 0) a.stats[4] = s_status;
        drain_weights();
        return;
    }
    const double dx = a.dx, dy = a.dy;
    const R dt = (R)a.c.dt;
    const bool unit_dt = (a.c.dt == 1.0);  // x / 1.0 == x exactly: skip the division
    R* bfs = a.scratch;                       // 9 * NB post-streaming populations (DFC)
    R* dfl = a.scratch + 9 * (size_t)NB;      // 9 * Lb distribution corrections (DFC)
    int* cfill = a.iscratch;                  // NB

    // ---- markers of this step (overlaps the bulk copy) ----------------------
    for (int l = tid; l < Lb; l += IBM_THREADS) {
        double x, y, vx, vy;
        if (a.xt_table) {
            // iblbm/physics/motion.py:44-50: Lx = Lx_c - xt, desired velocity (xt, 0)
            const double xt = a.xt_table[s_step];
            x = a.Lx_c[l] - xt;
            y = a.Ly_c[l];
            vx = xt;
            vy = 0.0;
        } else {
            x = a.Lx[l];
            y = a.Ly[l];
            vx = a.dvel[2 * l];
            vy = a.dvel[2 * l + 1];
            if (a.dvel_scale) {  // the Taylor-Green markers' analytic decay
                const double d = *a.dvel_scale;
                vx = vx * d;
                vy = vy * d;
            }
        }
        sh.dvx[l] = (R)vx;
        sh.dvy[l] = (R)vy;
        sh.Lux[l] = 0; sh.Luy[l] = 0; sh.Lfx[l] = 0; sh.Lfy[l] = 0; sh.R_[l] = 0;
        if (rebuild) {
            int p = 0;
            while (p + 1 < P && l >= a.moff[p + 1]) ++p;
            sh.part[l] = p;
            // iblbm/ibm/df.py:94-114: nearest node and separable weights
            const double fxr = floor(x / dx + 0.5), fyr = floor(y / dy + 0.5);
            const long long ix0 = (long long)fmin(fmax(fxr, -1.0e9), 1.0e9);
            const long long iy0 = (long long)fmin(fmax(fyr, -1.0e9), 1.0e9);
            sh.ix0[l] = (int)ix0;
            sh.iy0[l] = (int)iy0;
#pragma unroll
            for (int d = -A; d <= A; ++d) {
                sh.wx[l * 5 + d + A] = (R)phi(A == 2 ? 0 : 1, (x - (double)(ix0 + d) * dx) / dx);
                sh.wy[l * 5 + d + A] = (R)phi(A == 2 ? 0 : 1, (y - (double)(iy0 + d) * dy) / dy);
            }
        }
    }

    int nb;
    if (rebuild) {
        __syncthreads();
        auto node_of = [&](int l, int k) -> long long {
            const int ei = min(max(sh.ix0[l] + k / SW - A, 0), g.nx - 1);
            const int ej = min(max(sh.iy0[l] + k % SW - A, 0), g.ny - 1);
            return (long long)ej * g.nx + ei;
        };
        // ---- band rebuild ------------------------------------------------------
        if (tid == 0) { s_box[0] = INT_MAX; s_box[1] = INT_MAX; s_box[2] = INT_MIN; s_box[3] = INT_MIN; }
        const int nprev = *a.band_count;
        __syncthreads();
        for (int l = tid; l < Lb; l += IBM_THREADS) {
            atomicMin(&s_box[0], min(max(sh.ix0[l] - A, 0), g.nx - 1));
            atomicMin(&s_box[1], min(max(sh.iy0[l] - A, 0), g.ny - 1));
            atomicMax(&s_box[2], min(max(sh.ix0[l] + A, 0), g.nx - 1));
            atomicMax(&s_box[3], min(max(sh.iy0[l] + A, 0), g.ny - 1));
        }
        for (int b = tid; b < nprev; b += IBM_THREADS) a.map[a.band_nodes[b]] = -1;  // clear the previous band
        __syncthreads();
        const int bx0 = s_box[0], by0 = s_box[1], bw = s_box[2] - s_box[0] + 1, bh = s_box[3] - s_box[1] + 1;
        for (int e = tid; e < S * Lb; e += IBM_THREADS) a.map[node_of(e % Lb, e / Lb)] = -2;
        __syncthreads();
        const int cells = bw * bh;
        const int chunk = (cells + IBM_THREADS - 1) / IBM_THREADS;
        const int c0 = tid * chunk, c1 = min(c0 + chunk, cells);
        int cnt = 0;
        for (int c = c0; c < c1; ++c) cnt += (a.map[(long long)(by0 + c / bw) * g.nx + bx0 + c % bw] == -2);
        int total;
        int idx = block_exscan(cnt, sh.ired, &total);
        if (total > NB) {
            if (tid == 0) s_status = ST_BAND_CAPACITY;
        } else {
            for (int c = c0; c < c1; ++c) {
                const long long n = (long long)(by0 + c / bw) * g.nx + bx0 + c % bw;
                if (a.map[n] == -2) {
                    a.map[n] = idx;
                    a.band_nodes[idx] = (int)n;
                    sh.nodes[idx] = (int)n;
                    ++idx;
                }
            }
        }
        __syncthreads();
        if (s_status != ST_OK) {
            // leave a consistent empty band: unmark every node this step marked
            for (int e = tid; e < S * Lb; e += IBM_THREADS) a.map[node_of(e % Lb, e / Lb)] = -1;
            if (tid == 0) {
                a.stats[4] = s_status;
                *a.band_count = 0;
                a.box[0] = 0; a.box[1] = 0; a.box[2] = 0; a.box[3] = 0;
            }
            drain_weights();
            return;
        }
        nb = total;
        if (tid == 0) {
            *a.band_count = nb;
            a.box[0] = bx0; a.box[1] = by0; a.box[2] = bw; a.box[3] = bh;
        }
        // slot -> band index, list counts
        for (int b = tid; b < nb; b += IBM_THREADS) cfill[b] = 0;
        __syncthreads();
        for (int e = tid; e < S * Lb; e += IBM_THREADS) {
            const int l = e % Lb, k = e / Lb;
            const int b = a.map[node_of(l, k)];
            sh.sidx[l * S + k] = b;
            atomicAdd(&cfill[b], 1);
        }
        __syncthreads();
        {
            const int ch = (nb + IBM_THREADS - 1) / IBM_THREADS;
            const int b0 = tid * ch, b1 = min(b0 + ch, nb);
            int c = 0;
            for (int b = b0; b < b1; ++b) c += cfill[b];
            int tot;
            int base = block_exscan(c, sh.ired, &tot);
            for (int b = b0; b < b1; ++b) { sh.cstart[b] = base; base += cfill[b]; cfill[b] = 0; }
            if (tid == 0) sh.cstart[nb] = tot;
        }
        __syncthreads();
        for (int e = tid; e < S * Lb; e += IBM_THREADS) {
            const int l = e % Lb, k = e / Lb;
            const int b = sh.sidx[l * S + k];
            sh.ent[sh.cstart[b] + atomicAdd(&cfill[b], 1)] = (l << 5) | k;
        }
        __syncthreads();
        // order each list by (k, l): the reference's scatter order; then the
        // entries' spreading weights (wx*wy)*ds of their particle
        for (int b = tid; b < nb; b += IBM_THREADS) {
            const int s0 = sh.cstart[b], s1 = sh.cstart[b + 1];
            for (int u = s0 + 1; u < s1; ++u) {
                const int v = sh.ent[u];
                const int kv = v & 31, lv = v >> 5;
                int w = u - 1;
                while (w >= s0) {
                    const int c = sh.ent[w];
                    const int kc = c & 31, lc = c >> 5;
                    if (kc < kv || (kc == kv && lc < lv)) break;
                    sh.ent[w + 1] = c;
                    --w;
                }
                sh.ent[w + 1] = v;
            }
            for (int u = s0; u < s1; ++u) {
                const int e = sh.ent[u], l = e >> 5;
                sh.entw[u] = wgt<A>(sh, l, e & 31) * (R)a.larea[sh.part[l]];
            }
        }
        __syncthreads();
        if (!GS && !a.xt_table) {
            // cache the per-step-constant block for the following steps
            const int4* s4 = reinterpret_cast<const int4*>(smem_raw);
            int4* d4 = reinterpret_cast<int4*>(a.list_cache);
            for (size_t u = tid; u < Lay.static_bytes / 16; u += IBM_THREADS) d4[u] = s4[u];
        }
        if (tid == 0) s_nb = nb;
        __syncthreads();
    } else {
        // wait for the bulk copy (bounded: a copy that does not land is reported)
        bool done = GS;
        for (long long it = 0; it < wait_limit && !done; ++it) done = mbar_try_wait(&s_bar, 0);
        if (!done) {
            if (tid == 0) s_status = ST_COPY_TIMEOUT;
            for (long long it = 0; it < wait_limit && !done; ++it) done = mbar_try_wait(&s_bar, 0);
        }
        __syncthreads();
        if (s_status != ST_OK) {
            if (tid == 0) a.stats[4] = s_status;
            drain_weights();
            return;
        }
        nb = s_nb;
    }

    // ---- exclusion boxes: this step's (checked) and the next step's ------------
    if (tid == 0) {
        const int x0 = s_box[0], y0 = s_box[1], x1 = s_box[2], y1 = s_box[3];
        if (a.excl_cur) {
            const int* e = a.excl_cur;
            if (x0 < e[0] || y0 < e[1] || x1 >= e[0] + e[2] || y1 >= e[1] + e[3]) s_status = ST_EXCL;
        }
        if (a.excl_next) {
            const int ex0 = max(x0 - 1, 0), ey0 = max(y0 - 1, 0);
            const int ex1 = min(x1 + 1, g.nx - 1), ey1 = min(y1 + 1, g.ny - 1);
            a.excl_next[0] = ex0;
            a.excl_next[1] = ey0;
            a.excl_next[2] = ex1 - ex0 + 1;
            a.excl_next[3] = ey1 - ey0 + 1;
        }
    }

    // ---- post-streaming populations and moments on the band ------------------------
    R* fs_keep = (METHOD == IBM_DFC) ? bfs : nullptr;
    if (a.field_ro || a.field_fstar) {
        field_moments(a, nb, sh, fs_keep);
    } else switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN: band_moments<SHIFTED, BC_DIRICHLET_NEUMANN>(a, g, bc, nb, sh, fs_keep); break;
    case BC_OPEN: band_moments<SHIFTED, BC_OPEN>(a, g, bc, nb, sh, fs_keep); break;
    case BC_SETTLING: band_moments<SHIFTED, BC_SETTLING>(a, g, bc, nb, sh, fs_keep); break;
    case BC_TG: band_moments<SHIFTED, BC_TG>(a, g, bc, nb, sh, fs_keep); break;
    default: band_moments<SHIFTED, BC_VELOCITY_INLET>(a, g, bc, nb, sh, fs_keep); break;
    }
    __syncthreads();

    const size_t pstride = 2 * (size_t)NB;
    if (METHOD == IBM_DF) {
        // iblbm/ibm/df.py:93-154, summed over particles as ibm/multi_particle.py:404-421
        const bool incomp = a.c.incompressible != 0;
        for (int l = tid; l < Lb && a.df_given_force; l += IBM_THREADS) {
            // the marker forces are given: only their spreading (Lux, Luy stay 0)
            sh.Lfx[l] = (R)a.Lfx[l];
            sh.Lfy[l] = (R)a.Lfy[l];
        }
        for (int l = tid; l < Lb && !a.df_given_force; l += IBM_THREADS) {
            R Rl, ux, uy;
            {
                R dummy;
                interp2<A>(sh, sh.bro, sh.bro, l, Rl, dummy);
            }
            interp2<A>(sh, sh.bwx, sh.bwy, l, ux, uy);
            sh.R_[l] = Rl; sh.Lux[l] = ux; sh.Luy[l] = uy;
            R fx, fy;
            if (incomp) { fx = (R)2 * (sh.dvx[l] - ux); fy = (R)2 * (sh.dvy[l] - uy); }
            else { fx = (R)2 * Rl * (sh.dvx[l] - ux); fy = (R)2 * Rl * (sh.dvy[l] - uy); }
            sh.Lfx[l] = unit_dt ? fx : fx / dt;
            sh.Lfy[l] = unit_dt ? fy : fy / dt;
        }
        __syncthreads();
        for (int b = tid; b < nb; b += IBM_THREADS) {
            const int u0 = sh.cstart[b], u1 = sh.cstart[b + 1];
            R tx = 0, ty = 0;
            if (P == 1) {
                spread2(sh, sh.Lfx, sh.Lfy, u0, u1, tx, ty);
                if (a.band_fib_part) { a.band_fib_part[2 * b] = tx; a.band_fib_part[2 * b + 1] = ty; }
                tx = (R)0 + tx;
                ty = (R)0 + ty;
            } else {
                for (int p = 0; p < P; ++p) {
                    R ax = 0, ay = 0;
                    for (int u = u0; u < u1; ++u) {
                        const int l = sh.ent[u] >> 5;
                        if (sh.part[l] != p) continue;
                        ax += sh.Lfx[l] * sh.entw[u];
                        ay += sh.Lfy[l] * sh.entw[u];
                    }
                    if (a.band_fib_part) {
                        a.band_fib_part[p * pstride + 2 * b] = ax;
                        a.band_fib_part[p * pstride + 2 * b + 1] = ay;
                    }
                    tx += ax;
                    ty += ay;
                }
            }
            a.band_fib[2 * b] = tx;
            a.band_fib[2 * b + 1] = ty;
        }
    } else if (METHOD == IBM_MDF) {
        // iblbm/ibm/mdf.py:61-229 (one body) and iblbm/ibm/multi_particle.py:62-316 (coupled).
        // Each thread owns up to NPT band nodes (accumulators in registers) and at
        // most one marker (its slot -> band map and separable weights in registers).
        const bool incomp = COUPLED && a.c.incompressible != 0;  // mdf.py always uses the compressible law
        R vs[NPT], ftx[NPT], fty[NPT];
        int slot_node[NPT];  // the band node of each accumulator slot (-1: none)
#pragma unroll
        for (int jn = 0; jn < NPT; ++jn) {
            const int b = tid + jn * IBM_THREADS;
            slot_node[jn] = b < nb ? b : -1;
            vs[jn] = b < nb ? dt / ((R)2 * sh.bro[b]) : (R)0;
            ftx[jn] = 0;
            fty[jn] = 0;
            if (COUPLED && b < nb && a.band_fib_part)
                for (int p = 0; p < P; ++p) {
                    a.band_fib_part[p * pstride + 2 * b] = 0;
                    a.band_fib_part[p * pstride + 2 * b + 1] = 0;
                }
        }
        const bool own = tid < Lb;  // Lb <= IBM_THREADS (checked on the host)
        const int lo = own ? tid : 0;
        int hb[S];
        R hwx[SW], hwy[SW];
#pragma unroll
        for (int k = 0; k < S; ++k) hb[k] = sh.sidx[lo * S + k];
#pragma unroll
        for (int d = 0; d < SW; ++d) { hwx[d] = sh.wx[lo * 5 + d]; hwy[d] = sh.wy[lo * 5 + d]; }
        const R dvx = sh.dvx[lo], dvy = sh.dvy[lo];
        const int pl = COUPLED ? sh.part[lo] : 0;
        R Rl = 0;
        if (own) {
#pragma unroll
            for (int k = 0; k < S; ++k) Rl += sh.bro[hb[k]] * (hwx[k / SW] * hwy[k % SW]);
            sh.R_[lo] = Rl;
        }
        // ---- learned warm start (FP32 form, one body) ---------------------------------
        // Features of each marker before any correction; with bit 2 of mlp_mode the
        // network predicts the marker's converged force sum_it omega Lf, which is
        // spread and applied before the first iteration; with bit 1 the features
        // and the force actually accumulated are written out as training pairs.
        R mlp_gx = 0, mlp_gy = 0;
        bool mlp_rec = false;
        if constexpr (SHIFTED && !COUPLED) {
            const int mode = a.mlp_mode;
            mlp_rec = (mode & 1) != 0;
            const bool warm = (mode & 2) != 0;
            if (mode) {
                float* mA = reinterpret_cast<float*>(smem_raw + dyn_end);
                float* mB = mA + MLP_CHUNK * MLP_LD;
                float* mY = mB + MLP_CHUNK * MLP_LD;
                float* mGx = mY + MLP_CHUNK * 2;
                float* mGy = mGx + Lb;
                float* mWb = mGy + 3 * Lb;  // one hidden layer's weights (after the slips mSx, mSy)
                const float* Pm = reinterpret_cast<const float*>(smem_raw + dyn_end + mlp_act_bytes(Lb));
                bool use_net = false;
                if (warm) {
                    // a copy that does not land leaves this step on plain MDF
                    const bool ok = mbar_wait_bounded(&s_wbar, 0, wait_limit);
                    use_net = __syncthreads_and(ok) != 0;
                }
                const float inv_u = 1.0f / a.mlp_uref;
                // every marker's slip first: the features include the neighbours' slips
                float* mSx = mGy + Lb;
                float* mSy = mSx + Lb;
                if (own) {
                    R ux = 0, uy = 0;
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        const R w = hwx[k / SW] * hwy[k % SW];
                        ux += sh.bwx[hb[k]] * w;
                        uy += sh.bwy[hb[k]] * w;
                    }
                    mSx[lo] = (dvx - ux) * inv_u;
                    mSy[lo] = (dvy - uy) * inv_u;
                }
                __syncthreads();
                for (int c0 = 0; c0 < Lb; c0 += MLP_CHUNK) {
                    const int rows = min(MLP_CHUNK, Lb - c0);
                    if (own && lo >= c0 && lo < c0 + rows) {
                        float* row = mA + (lo - c0) * MLP_LD;
                        float* grow = mlp_rec ? a.mlp_features + (size_t)lo * 64 : nullptr;
                        auto put = [&](int i, float v) {
                            if (grow) grow[i] = v;
                            if (use_net) row[i] = (v - Pm[i]) * Pm[64 + i];
                        };
#pragma unroll 1
                        for (int k = 0; k < S; ++k) {
                            const int bk = sh.sidx[lo * S + k];
                            put(2 + 2 * k, sh.bwx[bk] * inv_u);
                            put(3 + 2 * k, sh.bwy[bk] * inv_u);
                        }
                        for (int k = S; k < 25; ++k) { put(2 + 2 * k, 0.0f); put(3 + 2 * k, 0.0f); }
                        put(0, mSx[lo]);
                        put(1, mSy[lo]);
                        double x, y;
                        if (a.xt_table) { x = a.Lx_c[lo] - a.xt_table[s_step]; y = a.Ly_c[lo]; }
                        else { x = a.Lx[lo]; y = a.Ly[lo]; }
                        put(52, (float)(x / dx - floor(x / dx + 0.5)));
                        put(53, (float)(y / dy - floor(y / dy + 0.5)));
                        const int p = sh.part[lo], m0 = a.moff[p], m1 = a.moff[p + 1];
                        const int nm = max(m1 - m0, 1);
                        const int lp = m0 + (lo - m0 + 1) % nm, lm = m0 + (lo - m0 + nm - 1) % nm;
                        float sn, cs;
                        sincosf(6.283185307179586f * (float)(lo - m0) / (float)max(m1 - m0, 1), &sn, &cs);
                        put(54, cs);
                        put(55, sn);
                        put(56, A == 2 ? 1.0f : 0.0f);
                        put(57, a.mlp_re * 0.01f);
                        put(58, (Rl - 1.0f) * 100.0f);
                        // slips of the two neighbouring markers on the body
                        put(59, mSx[lp]);
                        put(60, mSy[lp]);
                        put(61, mSx[lm]);
                        put(62, mSy[lm]);
                        put(63, 0.0f);
                    }
                    __syncthreads();
                    if (use_net) {
                        mlp_forward_tile<IBM_THREADS>(a.mlp_params, mA, mB, mY, rows, mWb);
                        if (own && lo >= c0 && lo < c0 + rows) {
                            mGx[lo] = mY[(lo - c0) * 2] / Pm[128];
                            mGy[lo] = mY[(lo - c0) * 2 + 1] / Pm[129];
                        }
                        __syncthreads();
                    }
                }
                if (use_net) {
                    // spread the predicted forces and correct the working velocity
#pragma unroll
                    for (int jn = 0; jn < NPT; ++jn) {
                        const int b = tid + jn * IBM_THREADS;
                        if (b < nb) {
                            R tx, ty;
                            spread2(sh, mGx, mGy, sh.cstart[b], sh.cstart[b + 1], tx, ty);
                            ftx[jn] += tx;
                            fty[jn] += ty;
                            sh.bwx[b] += tx * vs[jn];
                            sh.bwy[b] += ty * vs[jn];
                        }
                    }
                    if (own) { mlp_gx = mGx[lo]; mlp_gy = mGy[lo]; }
                    __syncthreads();
                }
            }
        }
        R lfx = 0, lfy = 0;
        const int min_iter = max(1, min(a.mdf_min_iterations, a.mdf_iterations));
        double omega_d = a.mdf_omega, omega_min = 0.0;
        if (COUPLED) {
            omega_d = fmin(a.mdf_omega * 0.8, a.mdf_omega_max);
            omega_min = omega_d * 0.125;
        }
        double prev = INFINITY, last = INFINITY;
        int iter_count = 0, diverged = 0, converged = 0, guard = 0;
        __syncthreads();
        // marker space (FP32 form, one body): set once the coupling matrix is built
        bool marker_space = false;
        float* msA = nullptr;
        float* msG = nullptr;
        R u0x = 0, u0y = 0;
        if constexpr (SHIFTED && !COUPLED) {
            // ---- marker-space iterations (FP32 form, one body) ---------------------
            // An iteration changes the working velocity at the band nodes by
            // vs * spread(omega Lf), so marker l's interpolated velocity is
            // u_l = u0_l + sum_m A_lm G_m, with G_m the force marker m has
            // accumulated (sum of omega Lf) and
            // A_lm = sum over the nodes both stencils cover of W_l vs W_m ds_m.
            // A is built once per step (banded: markers couple only to their
            // neighbours on the body), the iterations run on the markers alone
            // (one barrier of the marker-owning warps each), and the accumulated
            // forces are spread to the nodes once.  The operator is the node-space
            // loop's; that loop stays for coupled bodies, for marker sets that do
            // not fit, and wherever the overlaps do not account for every entry of
            // the node lists.
            const size_t off = dyn_end + (a.mlp_mode ? mlp_smem_bytes(Lb) : 0);
            if (ms_fits(off, Lb, S)) {
                msA = reinterpret_cast<float*>(smem_raw + off);
                float* msP = msA + (size_t)Lb * MS_W;  // W_lk vs(b_k) per stencil slot, while A is built
                msG = msP;  // then [2 buffers][x, y][MS_D + Lb + MS_D]: accumulated force with ring halos
                __shared__ R s_la[MAXP];
                if (tid < P) s_la[tid] = (R)a.larea[tid];
                for (int e = tid; e < Lb * S; e += IBM_THREADS) {
                    const int l = e / S, k = e - l * S;
                    msP[e] = wgt<A>(sh, l, k) * (dt / ((R)2 * sh.bro[sh.sidx[e]]));
                }
                __syncthreads();
                // slot i of marker m covers the lattice column of slot i + ox of
                // marker l, ox = ix0_m - ix0_l (rows alike): A_lm sums W_l vs over
                // the overlap of the two stencils times m's entry weight (wx wy) ds.
                // Entries in j-major order (a warp shares the neighbour offset),
                // each over the full SW x SW slot grid with slots outside the
                // overlap weighted 0 (loads clamped in bounds).
                for (int e = tid; e < Lb * MS_W; e += IBM_THREADS) {
                    const int j = e / Lb, l = e - j * Lb;
                    const int m = ms_ring(l + j - MS_D, Lb);
                    const int ox = sh.ix0[m] - sh.ix0[l], oy = sh.iy0[m] - sh.iy0[l];
                    R acc = 0;
                    if (ox > -SW && ox < SW && oy > -SW && oy < SW) {
                        const R La = s_la[sh.part[m]];
                        const float* pl = msP + (size_t)l * S;
                        R wym[SW];
#pragma unroll
                        for (int jj = 0; jj < SW; ++jj) {
                            const int t = jj - oy;
                            const R w = sh.wy[m * 5 + min(max(t, 0), SW - 1)];
                            wym[jj] = (t >= 0 && t < SW) ? w : (R)0;
                        }
#pragma unroll 1
                        for (int i = 0; i < SW; ++i) {
                            const int t = i - ox;
                            const R wxm = sh.wx[m * 5 + min(max(t, 0), SW - 1)];
                            const bool in = t >= 0 && t < SW;
#pragma unroll
                            for (int jj = 0; jj < SW; ++jj) {
                                const R ew = in ? (wxm * wym[jj]) * La : (R)0;
                                acc += pl[i * SW + jj] * ew;
                            }
                        }
                    }
                    msA[l * MS_W + j] = acc;
                }
                // the overlaps must account for every entry of the lists at marker
                // l's nodes (a marker further along the body, or stencil slots
                // clamped onto one edge node, are not covered by A)
                int over = 0;
                if (own) {
                    int n_list = 0, n_geo = 0;
#pragma unroll SW
                    for (int k = 0; k < S; ++k) {
                        const int b = sh.sidx[lo * S + k];
                        const R w = wgt<A>(sh, lo, k);
                        u0x += sh.bwx[b] * w;
                        u0y += sh.bwy[b] * w;
                        n_list += sh.cstart[b + 1] - sh.cstart[b];
                    }
                    const int x0 = sh.ix0[lo], y0 = sh.iy0[lo];
#pragma unroll
                    for (int j = 0; j < MS_W; ++j) {
                        const int m = ms_ring(lo + j - MS_D, Lb);
                        const int ox = abs(sh.ix0[m] - x0), oy = abs(sh.iy0[m] - y0);
                        if (ox < SW && oy < SW) n_geo += (SW - ox) * (SW - oy);
                    }
                    over = n_list != n_geo;
                }
                marker_space = !__syncthreads_or(over);
            }
        }
        // the restructured node-space loop (FP64, one body): when its room fits
        // and no node's list is longer than the stencil (lists of clamped edge
        // nodes can be; they take the plain loop)
        bool nsf = false;
        if constexpr (!SHIFTED && !COUPLED && !GS) {
            if (nsf_fits(Lay.total, Lb, NB, S)) {
                int mx = 0;
                for (int b = tid; b < nb; b += IBM_THREADS) mx = max(mx, sh.cstart[b + 1] - sh.cstart[b]);
                nsf = !__syncthreads_or(mx > S);
            }
        }
        if (marker_space) {
            if constexpr (SHIFTED && !COUPLED) {
                // MDF iterations on the markers: u_l = u0_l + sum_j A_l,j G_(l+j-MS_D)
                const int LH = Lb + 2 * MS_D;
                for (int e = tid; e < 4 * LH; e += IBM_THREADS) msG[e] = 0.0f;
                R arow[MS_W];
#pragma unroll
                for (int j = 0; j < MS_W; ++j) arow[j] = own ? msA[lo * MS_W + j] : (R)0;
                __syncthreads();
                const int nthr = (Lb + 31) & ~31;  // the warps that own markers
                if (tid < nthr) {
                    const int nw = nthr >> 5;
                    int cur = 0;
                    R ux = 0, uy = 0;
                    for (int it = 0; it < a.mdf_iterations; ++it) {
                        const R omega = (R)omega_d;
                        const float* Gx = msG + cur * 2 * LH;  // marker m at Gx[m + MS_D]
                        const float* Gy = Gx + LH;
                        float* Nx = msG + (cur ^ 1) * 2 * LH;
                        float* Ny = Nx + LH;
                        // squared slip as its FP64 bit pattern (0 for lanes without a marker)
                        unsigned long long key = 0;
                        if (own) {
                            R sx0 = 0, sy0 = 0, sx1 = 0, sy1 = 0;  // two chains: even and odd j
#pragma unroll
                            for (int j = 0; j < MS_W; j += 2) {
                                sx0 += arow[j] * Gx[lo + j];
                                sy0 += arow[j] * Gy[lo + j];
                                if (j + 1 < MS_W) {
                                    sx1 += arow[j + 1] * Gx[lo + j + 1];
                                    sy1 += arow[j + 1] * Gy[lo + j + 1];
                                }
                            }
                            ux = u0x + (sx0 + sx1);
                            uy = u0y + (sy0 + sy1);
                            const double ex = (double)dvx - (double)ux, ey = (double)dvy - (double)uy;
                            key = (unsigned long long)__double_as_longlong(ex * ex + ey * ey);
                            const R fx = (R)2 * Rl * (dvx - ux), fy = (R)2 * Rl * (dvy - uy);
                            lfx = unit_dt ? fx : fx / dt;
                            lfy = unit_dt ? fy : fy / dt;
                            // next forces, kept only if this iteration is accepted
                            const R nx = Gx[lo + MS_D] + omega * lfx, ny = Gy[lo + MS_D] + omega * lfy;
                            Nx[lo + MS_D] = nx;
                            Ny[lo + MS_D] = ny;
                            if (lo < MS_D) { Nx[lo + Lb + MS_D] = nx; Ny[lo + Lb + MS_D] = ny; }
                            if (lo >= Lb - MS_D) { Nx[lo - Lb + MS_D] = nx; Ny[lo - Lb + MS_D] = ny; }
                        }
                        // residual = max_l sqrt(slip^2) = sqrt(max_l slip^2) (sqrt is monotone
                        // and correctly rounded); the max runs on the bit patterns
                        unsigned long long* wk = reinterpret_cast<unsigned long long*>(sh.wred) + (it & 1) * NWARP;
                        const unsigned long long wmax = warp_max_bits(key);
                        if (lane == 0) wk[wid] = wmax;
                        bar_sync_n(1, nthr);
                        const unsigned long long mk = warp_max_bits(lane < nw ? wk[lane] : 0ull);
                        const double residual = sqrt(__longlong_as_double((long long)mk));
                        last = residual;
                        if (it > 0 && residual > prev * 1.5) {
                            diverged = 1;
                            iter_count = it + 1;
                            break;
                        }
                        if (mlp_rec && own) {
                            mlp_gx += omega * lfx;
                            mlp_gy += omega * lfy;
                        }
                        cur ^= 1;
                        prev = residual;
                        iter_count = it + 1;
                        if ((it + 1) >= min_iter && residual < a.mdf_tol) {
                            converged = 1;
                            break;
                        }
                    }
                    if (own) {
                        sh.Lux[lo] = ux;
                        sh.Luy[lo] = uy;
                        sh.Lfx[lo] = lfx;
                        sh.Lfy[lo] = lfy;
                    }
                    if (tid == 0) s_cur = cur;
                }
                __syncthreads();
                guard = -1;  // reported in stats[3]: the iterations ran in marker space
                const float* Gx = msG + s_cur * 2 * LH + MS_D;
                const float* Gy = Gx + LH;
#pragma unroll
                for (int jn = 0; jn < NPT; ++jn) {
                    const int b = tid + jn * IBM_THREADS;
                    if (b < nb) {
                        R tx, ty;
                        spread2(sh, Gx, Gy, sh.cstart[b], sh.cstart[b + 1], tx, ty);
                        ftx[jn] += tx;
                        fty[jn] += ty;
                    }
                }
            }
        } else if (nsf) {
            if constexpr (!SHIFTED && !COUPLED && !GS) {
                char* xs = smem_raw + dyn_end;
                int* rk_node = reinterpret_cast<int*>(xs + nsf_stage_bytes(Lb, S));
                int* rk_len = rk_node + NB;
                int* jd_off = rk_len + NB;     // S + 2: list position j starts at jd_off[j]
                int* hist = jd_off + (S + 2);  // S + 2: nodes per list length
                int* cur = hist + (S + 2);     // S + 2: rank cursors per list length
                // ---- lists in jagged-diagonal order ---------------------------------
                if (tid < S + 2) hist[tid] = 0;
                __syncthreads();
                for (int b = tid; b < nb; b += IBM_THREADS) atomicAdd(&hist[sh.cstart[b + 1] - sh.cstart[b]], 1);
                __syncthreads();
                if (tid == 0) {
                    // ranks by decreasing length: nodes of length n start after every longer one
                    int acc = 0;
                    for (int n = S; n >= 0; --n) { cur[n] = acc; acc += hist[n]; }
                    // position j holds the nodes longer than j: ranks 0 .. cur[j] - 1
                    int off = 0;
                    for (int j = 0; j <= S; ++j) { jd_off[j] = off; off += cur[j]; }
                    jd_off[S + 1] = off;
                }
                __syncthreads();
                for (int b = tid; b < nb; b += IBM_THREADS) {
                    const int n = sh.cstart[b + 1] - sh.cstart[b];
                    const int r = atomicAdd(&cur[n], 1);  // any order within a length class
                    rk_node[r] = b;
                    rk_len[r] = n;
                }
                __syncthreads();
                int* jl = reinterpret_cast<int*>(xs);                                    // staging: marker of entry
                R* jw = reinterpret_cast<R*>(xs + up16(sizeof(int) * (size_t)Lb * S));  // staging: its weight
                for (int r = tid; r < nb; r += IBM_THREADS) {
                    const int b = rk_node[r], u0 = sh.cstart[b];
                    for (int j = 0; j < rk_len[r]; ++j) {
                        jl[jd_off[j] + r] = sh.ent[u0 + j] >> 5;
                        jw[jd_off[j] + r] = sh.entw[u0 + j];
                    }
                }
                __syncthreads();
                for (int u = tid; u < Lb * S; u += IBM_THREADS) {  // the plain lists are not read again this step
                    sh.ent[u] = jl[u];
                    sh.entw[u] = jw[u];
                }
                // ---- per thread: its accumulator slots (ranks) and its marker slots ----
#pragma unroll
                for (int jn = 0; jn < NPT; ++jn) {
                    const int r = tid + jn * IBM_THREADS;
                    slot_node[jn] = r < nb ? rk_node[r] : -1;
                    vs[jn] = r < nb ? dt / ((R)2 * sh.bro[rk_node[r]]) : (R)0;
                }
                __syncthreads();
                for (int it = 0; it < a.mdf_iterations; ++it) {
                    unsigned long long* wk = reinterpret_cast<unsigned long long*>(sh.wred) + (it & 1) * NWARP;
                    const R omega = (R)omega_d;
                    // phase A: interpolate the working velocity (one thread per marker, slots in
                    // order), squared slip, force
                    unsigned long long key = 0;  // squared slip as its bit pattern
                    if (own) {
                        R ux = 0, uy = 0;
#pragma unroll
                        for (int gi = 0; gi < SW; ++gi) {
                            R vx[SW], vy[SW];
#pragma unroll
                            for (int gj = 0; gj < SW; ++gj) {
                                const int bk = sh.sidx[lo * S + gi * SW + gj];
                                vx[gj] = sh.bwx[bk];
                                vy[gj] = sh.bwy[bk];
                            }
#pragma unroll
                            for (int gj = 0; gj < SW; ++gj) {
                                const R w = sh.wx[lo * 5 + gi] * sh.wy[lo * 5 + gj];
                                ux += vx[gj] * w;
                                uy += vy[gj] * w;
                            }
                        }
                        sh.Lux[lo] = ux;
                        sh.Luy[lo] = uy;
                        const double ex = (double)dvx - (double)ux, ey = (double)dvy - (double)uy;
                        key = (unsigned long long)__double_as_longlong(ex * ex + ey * ey);
                        const R fx = (R)2 * Rl * (dvx - ux), fy = (R)2 * Rl * (dvy - uy);
                        sh.Lfx[lo] = unit_dt ? fx : fx / dt;
                        sh.Lfy[lo] = unit_dt ? fy : fy / dt;
                    }
                    // residual = max_l sqrt(slip^2) = sqrt(max_l slip^2): sqrt is monotone and
                    // correctly rounded; the max runs on the bit patterns (NaN above all numbers)
                    const unsigned long long wmax = warp_max_bits(key);
                    if (lane == 0) wk[wid] = wmax;
                    __syncthreads();  // (a)
                    const double residual =
                        sqrt(__longlong_as_double((long long)warp_max_bits(lane < NWARP ? wk[lane] : 0ull)));
                    last = residual;
                    if (it > 0 && residual > prev * 1.5) {
                        diverged = 1;
                        iter_count = it + 1;
                        break;
                    }
                    // phase B: spread, relax, update the working velocity of the owned nodes
#pragma unroll
                    for (int jn = 0; jn < NPT; ++jn) {
                        const int r = tid + jn * IBM_THREADS;
                        if (r < nb) {
                            const int n = rk_len[r];
                            R ax = 0, ay = 0;
                            int j = 0;
                            for (; j + 4 <= n; j += 4) {
                                const int u0 = jd_off[j] + r, u1 = jd_off[j + 1] + r;
                                const int u2 = jd_off[j + 2] + r, u3 = jd_off[j + 3] + r;
                                const int l0 = sh.ent[u0], l1 = sh.ent[u1], l2 = sh.ent[u2], l3 = sh.ent[u3];
                                const R w0 = sh.entw[u0], w1 = sh.entw[u1], w2 = sh.entw[u2], w3 = sh.entw[u3];
                                const R p0 = sh.Lfx[l0] * w0, p1 = sh.Lfx[l1] * w1, p2 = sh.Lfx[l2] * w2,
                                        p3 = sh.Lfx[l3] * w3;
                                const R q0 = sh.Lfy[l0] * w0, q1 = sh.Lfy[l1] * w1, q2 = sh.Lfy[l2] * w2,
                                        q3 = sh.Lfy[l3] * w3;
                                ax += p0; ax += p1; ax += p2; ax += p3;
                                ay += q0; ay += q1; ay += q2; ay += q3;
                            }
                            for (; j < n; ++j) {
                                const int u = jd_off[j] + r;
                                const int l = sh.ent[u];
                                const R w = sh.entw[u];
                                ax += sh.Lfx[l] * w;
                                ay += sh.Lfy[l] * w;
                            }
                            const R tx = ax * omega, ty = ay * omega;
                            ftx[jn] += tx;
                            fty[jn] += ty;
                            const int b = slot_node[jn];
                            sh.bwx[b] += tx * vs[jn];
                            sh.bwy[b] += ty * vs[jn];
                        }
                    }
                    __syncthreads();  // (b)
                    prev = residual;
                    iter_count = it + 1;
                    if ((it + 1) >= min_iter && residual < a.mdf_tol) {
                        converged = 1;
                        break;
                    }
                }
            }
        } else {
            for (int it = 0; it < a.mdf_iterations; ++it) {
                double* wr = sh.wred + (it & 1) * MAXP * NWARP;
                const R omega = (R)omega_d;
                // phase A: interpolate the working velocity, slip residual, force
                double rl = -INFINITY;
                if (own) {
                    R ux = 0, uy = 0;
#pragma unroll
                    for (int gi = 0; gi < SW; ++gi) {  // one stencil row (di) at a time, slots in order
                        R vx[SW], vy[SW];
#pragma unroll
                        for (int gj = 0; gj < SW; ++gj) {
                            vx[gj] = sh.bwx[hb[gi * SW + gj]];
                            vy[gj] = sh.bwy[hb[gi * SW + gj]];
                        }
#pragma unroll
                        for (int gj = 0; gj < SW; ++gj) {
                            const R w = hwx[gi] * hwy[gj];
                            ux += vx[gj] * w;
                            uy += vy[gj] * w;
                        }
                    }
                    sh.Lux[lo] = ux;
                    sh.Luy[lo] = uy;
                    // slip norm in FP64 (exact differences of the R values)
                    const double ex = (double)dvx - (double)ux, ey = (double)dvy - (double)uy;
                    rl = sqrt(ex * ex + ey * ey);
                    R fx, fy;
                    if (incomp) { fx = (R)2 * (dvx - ux); fy = (R)2 * (dvy - uy); }
                    else { fx = (R)2 * Rl * (dvx - ux); fy = (R)2 * Rl * (dvy - uy); }
                    lfx = unit_dt ? fx : fx / dt;
                    lfy = unit_dt ? fy : fy / dt;
                    sh.Lfx[lo] = lfx;
                    sh.Lfy[lo] = lfy;
                }
                if (!COUPLED) {
                    const double v = warp_nanmax(rl);
                    if (lane == 0) wr[wid] = v;
                } else {
                    for (int p = 0; p < P; ++p) {
                        const double v = warp_nanmax((own && pl == p) ? rl : -INFINITY);
                        if (lane == 0) wr[p * NWARP + wid] = v;
                    }
                }
                __syncthreads();  // (a)
                double residual;
                if (!COUPLED) {
                    residual = -INFINITY;
#pragma unroll
                    for (int w = 0; w < NWARP; ++w) residual = nanmax(residual, wr[w]);
                } else {
                    residual = 0.0;  // Python max over the particles' numpy maxima, from 0.0
                    for (int p = 0; p < P; ++p) {
                        double rp = -INFINITY;
#pragma unroll
                        for (int w = 0; w < NWARP; ++w) rp = nanmax(rp, wr[p * NWARP + w]);
                        if (rp > residual) residual = rp;
                    }
                }
                last = residual;
                if (!COUPLED) {
                    if (it > 0 && residual > prev * 1.5) {
                        diverged = 1;
                        iter_count = it + 1;
                        break;
                    }
                } else if (it > 0 && residual > prev * 1.2) {
                    guard += 1;
                    omega_d = fmax(omega_d * 0.5, omega_min);
                    if (omega_d <= omega_min) {
                        diverged = 1;
                        break;
                    }
                    prev = residual;
                    continue;
                }
                if (mlp_rec && own) {
                    mlp_gx += omega * lfx;
                    mlp_gy += omega * lfy;
                }
                // phase B: spread, relax, update the working velocity of the owned nodes
#pragma unroll
                for (int jn = 0; jn < NPT; ++jn) {
                    const int b = tid + jn * IBM_THREADS;
                    if (b < nb) {
                        const int u0 = sh.cstart[b], u1 = sh.cstart[b + 1];
                        R tx, ty;
                        if (!COUPLED) {
                            R ax, ay;
                            spread2(sh, sh.Lfx, sh.Lfy, u0, u1, ax, ay);
                            tx = ax * omega;
                            ty = ay * omega;
                        } else {
                            tx = 0;
                            ty = 0;
                            for (int p = 0; p < P; ++p) {
                                R ax = 0, ay = 0;
                                for (int u = u0; u < u1; ++u) {
                                    const int l = sh.ent[u] >> 5;
                                    if (sh.part[l] != p) continue;
                                    ax += sh.Lfx[l] * sh.entw[u];
                                    ay += sh.Lfy[l] * sh.entw[u];
                                }
                                const R fx = ax * omega, fy = ay * omega;
                                if (a.band_fib_part) {
                                    a.band_fib_part[p * pstride + 2 * b] += fx;
                                    a.band_fib_part[p * pstride + 2 * b + 1] += fy;
                                }
                                tx += fx;
                                ty += fy;
                            }
                        }
                        ftx[jn] += tx;
                        fty[jn] += ty;
                        if (incomp) {
                            sh.bwx[b] += (R)0.5 * tx * dt;
                            sh.bwy[b] += (R)0.5 * ty * dt;
                        } else {
                            sh.bwx[b] += tx * vs[jn];
                            sh.bwy[b] += ty * vs[jn];
                        }
                    }
                }
                __syncthreads();  // (b)
                prev = residual;
                if (COUPLED) iter_count += 1;
                else iter_count = it + 1;
                if ((it + 1) >= min_iter && residual < a.mdf_tol) {
                    converged = 1;
                    break;
                }
            }
        }
#pragma unroll
        for (int jn = 0; jn < NPT; ++jn) {
            const int b = slot_node[jn];
            if (b >= 0) {
                a.band_fib[2 * b] = ftx[jn];
                a.band_fib[2 * b + 1] = fty[jn];
                if (!COUPLED && a.band_fib_part) {
                    a.band_fib_part[2 * b] = ftx[jn];
                    a.band_fib_part[2 * b + 1] = fty[jn];
                }
            }
        }
        if (tid == 0) {
            a.stats[0] = iter_count;
            a.stats[1] = diverged;
            a.stats[2] = converged;
            a.stats[3] = nsf ? -2 : guard;
            a.dstats[0] = last;
            a.dstats[1] = omega_d;
        }
        if constexpr (SHIFTED && !COUPLED) {
            if (mlp_rec && own) {
                a.mlp_targets[2 * lo] = mlp_gx;
                a.mlp_targets[2 * lo + 1] = mlp_gy;
            }
        }
    } else if (METHOD == IBM_DFC) {
        // iblbm/ibm/dfc.py: compute_lambda (126-186) unless cached, interpolate_f
        // (55-95), bounce_back_fi (98-123), spread_delta_f (189-229),
        // compute_dfc_fluid_force (232-253)
        const R La = (R)a.larea[0];
        const bool have = a.dfc_cache_lambda && a.lambda_valid && *a.lambda_valid;
        if (!have) {
            for (int b = tid; b < nb; b += IBM_THREADS) {
                R wt = 0;
                for (int u = sh.cstart[b]; u < sh.cstart[b + 1]; ++u) {
                    const int e = sh.ent[u];
                    wt += wgt<A>(sh, e >> 5, e & 31);
                }
                sh.bwx[b] = wt;  // W_total
            }
            __syncthreads();
            const R rho_f = a.dfc_rho_f > 0.0 ? (R)a.dfc_rho_f : (R)1;
            for (int l = tid; l < Lb; l += IBM_THREADS) {
                R ws, dummy;
                interp2<A>(sh, sh.bwx, sh.bwx, l, ws, dummy);
                a.lambda[l] = (R)1 / ((R)2 * rho_f * La * ws);
            }
            __syncthreads();
            if (tid == 0 && a.dfc_cache_lambda && a.lambda_valid) *a.lambda_valid = 1;
        }
        const R cs2 = (R)1 / (R)3;
        const R cscale = (R)a.correction_scale;
        for (int l = tid; l < Lb; l += IBM_THREADS) {
            R fi[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) fi[q] = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int b = sh.sidx[l * S + k];
                const R w = wgt<A>(sh, l, k);
#pragma unroll
                for (int q = 0; q < 9; ++q) fi[q] += bfs[9 * (size_t)b + q] * w;
            }
            const R lam = (R)a.lambda[l];
            R sx = 0, sy = 0;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const R edu = edot_r<R>(q, sh.dvx[l], sh.dvy[l]);
                const R fbb = fi[opp_(q)] + (R)2 * (R)w_(q) * (R)1 * edu / cs2;
                const R dev = fbb - fi[q];
                dfl[9 * (size_t)l + q] = cscale * lam * dev;
                const R s = -(lam * dev * La);
                sx += s * (R)ex_(q);
                sy += s * (R)ey_(q);
            }
            if (a.dfc_force) {
                a.dfc_force[2 * l] = cscale * sx;
                a.dfc_force[2 * l + 1] = cscale * sy;
            }
        }
        __syncthreads();
        for (int b = tid; b < nb; b += IBM_THREADS) {
            R acc[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] = 0;
            for (int u = sh.cstart[b]; u < sh.cstart[b + 1]; ++u) {
                const int l = sh.ent[u] >> 5;
                const R w = sh.entw[u];
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[q] += dfl[9 * (size_t)l + q] * w;
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) a.band_df[9 * (size_t)b + q] = acc[q];
        }
    }
    __syncthreads();
    for (int l = tid; l < Lb; l += IBM_THREADS) {
        if (a.Lux) a.Lux[l] = sh.Lux[l];
        if (a.Luy) a.Luy[l] = sh.Luy[l];
        if (a.Lfx) a.Lfx[l] = sh.Lfx[l];
        if (a.Lfy) a.Lfy[l] = sh.Lfy[l];
    }
    if (tid == 0) {
        a.stats[4] = s_status;
        if (a.step_counter) *a.step_counter = s_step + 1;
    }
}

template <class ARGS, typename R, bool SHIFTED, int A, int METHOD, bool COUPLED, bool GS>
__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_step_kernel(const ARGS a, BcOf<SHIFTED> bc)
{
    ibm_step_body<ARGS, R, SHIFTED, A, METHOD, COUPLED, GS>(a, bc);
}

// Many independent cases in one launch: CTA b runs the band step of case b,
// whose argument block it copies from global into shared memory first.  The
// stencil radius, method and coupling are per case (uniform over the CTA).
template <class ARGS, typename R, bool SHIFTED>
__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_batch_kernel(const ARGS* __restrict__ args)
{
    __shared__ __align__(16) ARGS sa;
    __shared__ BcOf<SHIFTED> sbc;
    {
        const int* src = reinterpret_cast<const int*>(args + blockIdx.x);
        int* dst = reinterpret_cast<int*>(&sa);
        for (int k = threadIdx.x; k < (int)(sizeof(ARGS) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) make_bc(sa.c, sbc);
    __syncthreads();
    const bool coupled = sa.method == IBM_MDF && sa.mdf_coupled;
    if (sa.delta_type == 0) {
        if (sa.method == IBM_DF) ibm_step_body<ARGS, R, SHIFTED, 2, IBM_DF, false>(sa, sbc);
        else if (sa.method == IBM_DFC) ibm_step_body<ARGS, R, SHIFTED, 2, IBM_DFC, false>(sa, sbc);
        else if (coupled) ibm_step_body<ARGS, R, SHIFTED, 2, IBM_MDF, true>(sa, sbc);
        else ibm_step_body<ARGS, R, SHIFTED, 2, IBM_MDF, false>(sa, sbc);
    } else {
        if (sa.method == IBM_DF) ibm_step_body<ARGS, R, SHIFTED, 1, IBM_DF, false>(sa, sbc);
        else if (sa.method == IBM_DFC) ibm_step_body<ARGS, R, SHIFTED, 1, IBM_DFC, false>(sa, sbc);
        else if (coupled) ibm_step_body<ARGS, R, SHIFTED, 1, IBM_MDF, true>(sa, sbc);
        else ibm_step_body<ARGS, R, SHIFTED, 1, IBM_MDF, false>(sa, sbc);
    }
}

// Launch one instantiation; the first launch of each sets its shared-memory limit.
template <class ARGS, class BCP, void (*K)(const ARGS, BCP)>
static cudaError_t launch_ibm(const ARGS& a, const BCP& bc, size_t smem, void* stream)
{
    const cudaError_t e = smem_limit_once<K>(IBM_SMEM_LIMIT);
    if (e != cudaSuccess) return e;
    K<<<1, IBM_THREADS, smem, (cudaStream_t)stream>>>(a, bc);
    return cudaGetLastError();
}

// Dynamic shared memory of one band step.
template <typename R, class ARGS>
static size_t ibm_smem(const ARGS& a, bool gs = false)
{
    const int S = a.delta_type == 0 ? 25 : 9;
    const Layout L = make_layout<R>(a.lb_total, a.band_capacity, S);
    size_t t = L.total - (gs ? L.static_bytes : 0);
    if (mlp_on(a)) t += mlp_smem_bytes(a.lb_total);
    if (ms_on(a) && ms_fits(t, a.lb_total, S)) t += ms_smem_bytes(a.lb_total, S);
    if (!gs && nsf_on(a) && nsf_fits(t, a.lb_total, a.band_capacity, S))
        t += nsf_smem_bytes(a.lb_total, a.band_capacity, S);
    return t;
}

inline bool mlp_args_ok(const iblbm_ibm_args&) { return true; }
inline bool mlp_args_ok(const iblbm_ibm32_args& a)
{
    if (!mlp_on(a)) return true;
    if (a.mlp_mode & ~3) return false;
    if ((a.mlp_mode & 2) && (!a.mlp_params || (reinterpret_cast<uintptr_t>(a.mlp_params) & 15))) return false;
    if ((a.mlp_mode & 1) && (!a.mlp_features || !a.mlp_targets)) return false;
    return a.mlp_uref > 0.0f;
}

// Whether a band step keeps its per-step-constant block in global memory: only
// when the whole layout does not fit in shared memory.
template <typename R, class ARGS>
static bool ibm_global_static(const ARGS& a)
{
    return ibm_smem<R>(a) > (size_t)IBM_SMEM_LIMIT;
}

// Argument checks shared by both forms; returns IBLBM_OK or an error code.
// allow_gs: the caller can launch the global-static form (single-case launches).
template <typename R, class ARGS>
static int check_ibm_args(const ARGS* a, bool allow_gs = false)
{
    if (!a) return IBLBM_E_ARG;
    const bool fields = a->field_ro || a->field_fstar;
    if (fields && (a->method == IBM_DFC ? !a->field_fstar : (!a->field_ro || !a->field_ux || !a->field_uy)))
        return IBLBM_E_ARG;
    if (!a->moff || a->n_particles < 1 || a->n_particles > MAXP || a->lb_total < 1 || (!a->fpost_prev && !fields) ||
        !a->box || !a->map || !a->band_nodes || !a->band_count || !a->scratch || !a->iscratch || !a->stats ||
        !a->dstats || !a->larea || !a->list_cache)
        return IBLBM_E_ARG;
    if (a->delta_type != 0 && a->delta_type != 1) return IBLBM_E_ARG;
    if (a->method != IBM_DF && a->method != IBM_MDF && a->method != IBM_DFC) return IBLBM_E_ARG;
    if ((a->method == IBM_DF || a->method == IBM_MDF) && !a->band_fib) return IBLBM_E_ARG;
    if (a->df_given_force && (a->method != IBM_DF || !a->Lfx || !a->Lfy)) return IBLBM_E_ARG;
    if (a->method == IBM_DFC && (!a->band_df || !a->lambda || a->n_particles != 1)) return IBLBM_E_ARG;
    if (!a->xt_table && (!a->Lx || !a->Ly || !a->dvel)) return IBLBM_E_ARG;
    if (a->xt_table && (!a->Lx_c || !a->Ly_c || !a->step_counter || a->xt_len < 1)) return IBLBM_E_ARG;
    if (!fields && (a->c.bc == BC_OPEN || a->c.bc == BC_VELOCITY_INLET) && !a->uring_prev) return IBLBM_E_ARG;
    if (!fields && a->c.bc == BC_TG && (!a->c.tg_face || !a->c.tg_decay)) return IBLBM_E_ARG;
    if (a->c.bc < BC_DIRICHLET_NEUMANN || a->c.bc > BC_TG) return IBLBM_E_ARG;
    if (a->band_capacity < 1 || a->band_capacity > MAX_BAND || a->g.nx < 4 || a->g.ny < 4)
        return IBLBM_E_ARG;
    if ((long long)a->lb_total * 32 >= (1LL << 31)) return IBLBM_E_ARG;
    if ((reinterpret_cast<uintptr_t>(a->list_cache) & 15) != 0) return IBLBM_E_ARG;  // bulk-copy source
    if (ibm_smem<R>(*a) > (size_t)IBM_SMEM_LIMIT &&
        (!allow_gs || ibm_smem<R>(*a, true) > (size_t)IBM_SMEM_LIMIT))
        return IBLBM_E_CAPACITY;
    if (!mlp_args_ok(*a)) return IBLBM_E_ARG;
    if (a->method == IBM_MDF && a->lb_total > IBM_THREADS) return IBLBM_E_CAPACITY;
    return IBLBM_OK;
}

// Dispatch over (stencil radius, method, coupling).
template <class ARGS, typename R, bool SHIFTED>
static int dispatch_ibm(const ARGS* a, const BcOf<SHIFTED>& bc, void* stream)
{
    using BCP = BcOf<SHIFTED>;
    const bool gs = ibm_global_static<R>(*a);
    const size_t smem = ibm_smem<R>(*a, gs);
    const bool coupled = a->method == IBM_MDF && a->mdf_coupled;
    cudaError_t e = cudaErrorInvalidValue;
#define IBLBM_LAUNCH(AR, M, C)                                                                              \
    e = gs ? launch_ibm<ARGS, BCP, ibm_step_kernel<ARGS, R, SHIFTED, AR, M, C, true>>(*a, bc, smem, stream) \
           : launch_ibm<ARGS, BCP, ibm_step_kernel<ARGS, R, SHIFTED, AR, M, C, false>>(*a, bc, smem, stream)
    if (a->delta_type == 0) {
        if (a->method == IBM_DF) IBLBM_LAUNCH(2, IBM_DF, false);
        else if (a->method == IBM_DFC) IBLBM_LAUNCH(2, IBM_DFC, false);
        else if (coupled) IBLBM_LAUNCH(2, IBM_MDF, true);
        else IBLBM_LAUNCH(2, IBM_MDF, false);
    } else {
        if (a->method == IBM_DF) IBLBM_LAUNCH(1, IBM_DF, false);
        else if (a->method == IBM_DFC) IBLBM_LAUNCH(1, IBM_DFC, false);
        else if (coupled) IBLBM_LAUNCH(1, IBM_MDF, true);
        else IBLBM_LAUNCH(1, IBM_MDF, false);
    }
#undef IBLBM_LAUNCH
    if (e != cudaSuccess) return IBLBM_E_LAUNCH;
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

}  // namespace iblbm
