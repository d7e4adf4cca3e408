// ibm_f64.cu — immersed-boundary marker loop on the band, FP64.
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
//     weights, node list) is restored into shared memory from its global cache
//     with one TMA bulk copy (cp.async.bulk + mbarrier) while the marker data
//     loads; then post-streaming populations and moments on the band (the
//     dense kernel's device functions), and DF, MDF (every iteration resident
//     on chip: two barriers per iteration, residual reduced in shared memory,
//     no host round trip), coupled multi-particle MDF, or DFC.
//   exclusion box
//     the band's bounding box dilated by one node is written for the next
//     step: markers move less than one node per step, so the next band lies
//     inside it.  The bulk collide-stream kernel of the next step skips that
//     box and runs concurrently with this kernel; a small box kernel updates
//     the box once this kernel has produced the band forces.
//
// The kernel is latency-bound (one CTA, dependent FP64 sums in a fixed order):
// every loop over stencil slots or list entries is unrolled so its loads issue
// together and only the sum itself is serial.  All sums run in the reference's
// order, so results are bit-identical to the reference CPU path (-fmad=false).
#include <climits>
#include <cstdint>
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int IBM_THREADS = 512;
constexpr int NPT = 4;          // band nodes per thread in the MDF loop
constexpr int MAX_BAND = NPT * IBM_THREADS;  // band capacity limit (2048)
constexpr int MAXP = 8;    // particles per band kernel
constexpr int NWARP = IBM_THREADS / 32;
constexpr long long TMA_WAIT_LIMIT = 1LL << 22;

enum IbmStatus : int { ST_OK = 0, ST_BAND_CAPACITY = 1, ST_BOX_CAPACITY = 2, ST_MARKERS = 3, ST_TABLE = 4,
                       ST_EXCL = 5, ST_COPY_TIMEOUT = 6 };

template <int A>
struct Sten {
    static constexpr int SW = 2 * A + 1;
    static constexpr int S = SW * SW;
};

__host__ __device__ inline size_t up16(size_t x) { return (x + 15) & ~size_t(15); }

// Shared-memory layout.  The "static" block (everything a fixed body keeps
// between steps) is contiguous so that one bulk copy restores it.
struct Layout {
    size_t o_sidx, o_ent, o_cstart, o_nodes, o_part, o_wx, o_wy, o_entw, static_bytes;
    size_t o_dvx, o_dvy, o_R, o_Lux, o_Luy, o_Lfx, o_Lfy, o_bro, o_bwx, o_bwy, o_wred, o_ix0, o_iy0, o_ired, total;
};

__host__ __device__ inline Layout make_layout(int Lb, int NB, int S)
{
    Layout L;
    size_t o = 0;
    L.o_sidx = o; o = up16(o + sizeof(int) * (size_t)Lb * S);
    L.o_ent = o; o = up16(o + sizeof(int) * (size_t)Lb * S);
    L.o_cstart = o; o = up16(o + sizeof(int) * ((size_t)NB + 1));
    L.o_nodes = o; o = up16(o + sizeof(int) * (size_t)NB);
    L.o_part = o; o = up16(o + sizeof(int) * (size_t)Lb);
    L.o_wx = o; o = up16(o + sizeof(double) * (size_t)Lb * 5);
    L.o_wy = o; o = up16(o + sizeof(double) * (size_t)Lb * 5);
    L.o_entw = o; o = up16(o + sizeof(double) * (size_t)Lb * S);
    L.static_bytes = o;
    L.o_dvx = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_dvy = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_R = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_Lux = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_Luy = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_Lfx = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_Lfy = o; o = up16(o + sizeof(double) * (size_t)Lb);
    L.o_bro = o; o = up16(o + sizeof(double) * (size_t)NB);
    L.o_bwx = o; o = up16(o + sizeof(double) * (size_t)NB);
    L.o_bwy = o; o = up16(o + sizeof(double) * (size_t)NB);
    L.o_wred = o; o = up16(o + sizeof(double) * 2 * MAXP * NWARP);
    L.o_ix0 = o; o = up16(o + sizeof(int) * (size_t)Lb);
    L.o_iy0 = o; o = up16(o + sizeof(int) * (size_t)Lb);
    L.o_ired = o; o = up16(o + sizeof(int) * 64);
    L.total = o;
    return L;
}

struct Sm {
    int *sidx, *ent, *cstart, *nodes, *part, *ix0, *iy0, *ired;
    double *wx, *wy, *entw, *dvx, *dvy, *R, *Lux, *Luy, *Lfx, *Lfy, *bro, *bwx, *bwy, *wred;
};

__device__ inline Sm carve(char* base, const Layout& L)
{
    Sm s;
    s.sidx = reinterpret_cast<int*>(base + L.o_sidx);
    s.ent = reinterpret_cast<int*>(base + L.o_ent);
    s.cstart = reinterpret_cast<int*>(base + L.o_cstart);
    s.nodes = reinterpret_cast<int*>(base + L.o_nodes);
    s.part = reinterpret_cast<int*>(base + L.o_part);
    s.wx = reinterpret_cast<double*>(base + L.o_wx);
    s.wy = reinterpret_cast<double*>(base + L.o_wy);
    s.entw = reinterpret_cast<double*>(base + L.o_entw);
    s.dvx = reinterpret_cast<double*>(base + L.o_dvx);
    s.dvy = reinterpret_cast<double*>(base + L.o_dvy);
    s.R = reinterpret_cast<double*>(base + L.o_R);
    s.Lux = reinterpret_cast<double*>(base + L.o_Lux);
    s.Luy = reinterpret_cast<double*>(base + L.o_Luy);
    s.Lfx = reinterpret_cast<double*>(base + L.o_Lfx);
    s.Lfy = reinterpret_cast<double*>(base + L.o_Lfy);
    s.bro = reinterpret_cast<double*>(base + L.o_bro);
    s.bwx = reinterpret_cast<double*>(base + L.o_bwx);
    s.bwy = reinterpret_cast<double*>(base + L.o_bwy);
    s.wred = reinterpret_cast<double*>(base + L.o_wred);
    s.ix0 = reinterpret_cast<int*>(base + L.o_ix0);
    s.iy0 = reinterpret_cast<int*>(base + L.o_iy0);
    s.ired = reinterpret_cast<int*>(base + L.o_ired);
    return s;
}

// ---- TMA bulk copy global -> shared with an mbarrier ------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ double nanmax(double a, double b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ double warp_nanmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide exclusive scan of one int per thread; returns the prefix, writes the total.
__device__ int block_exscan(int v, int* ired, int* total)
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

// Post-streaming populations and moments of the band nodes; two nodes per pass
// so their global loads are in flight together.
template <int BC>
__device__ void band_moments(const iblbm_ibm_args& a, const Geom& g, const BcParams& bc, int nb, Sm& sh, double* bfs)
{
    const bool incomp = a.c.incompressible != 0;
    for (int b0 = threadIdx.x; b0 < nb; b0 += 2 * IBM_THREADS) {
        const int b1 = b0 + IBM_THREADS;
        const bool two = b1 < nb;
        const int n0 = sh.nodes[b0], n1 = sh.nodes[two ? b1 : b0];
        const int j0 = n0 / g.nx, i0 = n0 - j0 * g.nx, j1 = n1 / g.nx, i1 = n1 - j1 * g.nx;
        double f0[9], f1[9];
        fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i0, j0, f0);
        fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i1, j1, f1);
        double r0, x0, y0, r1, x1, y1;
        macro_seq(f0, incomp, r0, x0, y0);
        macro_seq(f1, incomp, r1, x1, y1);
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

template <int A>
__device__ __forceinline__ double wgt(const Sm& sh, int l, int k)
{
    constexpr int SW = Sten<A>::SW;
    return sh.wx[l * 5 + k / SW] * sh.wy[l * 5 + k % SW];
}

// Interpolate two band fields at marker l: (sum_k u[b_k] w_k, sum_k v[b_k] w_k)
// in slot order, loads issued together.
template <int A>
__device__ __forceinline__ void interp2(const Sm& sh, const double* u, const double* v, int l, double& su, double& sv)
{
    constexpr int S = Sten<A>::S;
    int bk[S];
    double wk[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        bk[k] = sh.sidx[l * S + k];
        wk[k] = wgt<A>(sh, l, k);
    }
    double x = 0.0, y = 0.0;
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
__device__ __forceinline__ void spread2(const Sm& sh, const double* gx, const double* gy, int u0, int u1,
                                        double& ax, double& ay)
{
    double x = 0.0, y = 0.0;
    int u = u0;
    for (; u + 4 <= u1; u += 4) {
        const int e0 = sh.ent[u], e1 = sh.ent[u + 1], e2 = sh.ent[u + 2], e3 = sh.ent[u + 3];
        const double w0 = sh.entw[u], w1 = sh.entw[u + 1], w2 = sh.entw[u + 2], w3 = sh.entw[u + 3];
        const int l0 = e0 >> 5, l1 = e1 >> 5, l2 = e2 >> 5, l3 = e3 >> 5;
        const double p0 = gx[l0] * w0, p1 = gx[l1] * w1, p2 = gx[l2] * w2, p3 = gx[l3] * w3;
        const double q0 = gy[l0] * w0, q1 = gy[l1] * w1, q2 = gy[l2] * w2, q3 = gy[l3] * w3;
        x += p0; x += p1; x += p2; x += p3;
        y += q0; y += q1; y += q2; y += q3;
    }
    for (; u < u1; ++u) {
        const int l = sh.ent[u] >> 5;
        const double w = sh.entw[u];
        x += gx[l] * w;
        y += gy[l] * w;
    }
    ax = x;
    ay = y;
}

template <int A, int METHOD, bool COUPLED>
__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_step_kernel(const iblbm_ibm_args a, BcParams bc)
{
    constexpr int SW = Sten<A>::SW, S = Sten<A>::S;
    extern __shared__ __align__(16) char smem_raw[];
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int P = a.n_particles, Lb = a.lb_total, NB = a.band_capacity;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const Layout Lay = make_layout(Lb, NB, S);
    Sm sh = carve(smem_raw, Lay);
    __shared__ int s_nb, s_status, s_box[4], s_step;
    __shared__ __align__(8) uint64_t s_bar;
    const bool rebuild = a.rebuild || a.xt_table;
    if (tid == 0) {
        s_status = ST_OK;
        s_step = a.step_counter ? *a.step_counter : 0;
        if (a.xt_table && (s_step < 0 || s_step >= a.xt_len)) s_status = ST_TABLE;
        if (!rebuild && s_status == ST_OK) {
            // restore the per-step-constant block of a fixed body in one bulk copy
            mbar_init(&s_bar);
            const uint32_t bytes = (uint32_t)Lay.static_bytes;
            mbar_expect(&s_bar, bytes);
            const char* src = reinterpret_cast<const char*>(a.list_cache);
            for (uint32_t off = 0; off < bytes; off += 65536u) {
                const uint32_t chunk = min(65536u, bytes - off);
                bulk_copy(smem_raw + off, src + off, chunk, &s_bar);
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
        return;
    }
    const double dx = a.dx, dy = a.dy, dt = a.c.dt;
    const bool unit_dt = (dt == 1.0);  // x / 1.0 == x exactly: skip the division
    double* bfs = a.scratch;                       // 9 * NB post-streaming populations (DFC)
    double* dfl = a.scratch + 9 * (size_t)NB;      // 9 * Lb distribution corrections (DFC)
    int* cfill = a.iscratch;                       // NB

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
        }
        sh.dvx[l] = vx;
        sh.dvy[l] = vy;
        sh.Lux[l] = 0.0; sh.Luy[l] = 0.0; sh.Lfx[l] = 0.0; sh.Lfy[l] = 0.0; sh.R[l] = 0.0;
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
                sh.wx[l * 5 + d + A] = phi(A == 2 ? 0 : 1, (x - (double)(ix0 + d) * dx) / dx);
                sh.wy[l * 5 + d + A] = phi(A == 2 ? 0 : 1, (y - (double)(iy0 + d) * dy) / dy);
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
                sh.entw[u] = wgt<A>(sh, l, e & 31) * a.larea[sh.part[l]];
            }
        }
        __syncthreads();
        if (!a.xt_table) {
            // cache the per-step-constant block for the following steps
            const int4* s4 = reinterpret_cast<const int4*>(smem_raw);
            int4* d4 = reinterpret_cast<int4*>(a.list_cache);
            for (size_t u = tid; u < Lay.static_bytes / 16; u += IBM_THREADS) d4[u] = s4[u];
        }
        if (tid == 0) s_nb = nb;
        __syncthreads();
    } else {
        // wait for the bulk copy (bounded: a copy that does not land is reported)
        bool done = false;
        for (long long it = 0; it < TMA_WAIT_LIMIT && !done; ++it) done = mbar_try_wait(&s_bar, 0);
        if (!done) {
            if (tid == 0) s_status = ST_COPY_TIMEOUT;
            for (long long it = 0; it < TMA_WAIT_LIMIT && !done; ++it) done = mbar_try_wait(&s_bar, 0);
        }
        __syncthreads();
        if (s_status != ST_OK) {
            if (tid == 0) a.stats[4] = s_status;
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
    double* fs_keep = (METHOD == IBM_DFC) ? bfs : nullptr;
    switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN: band_moments<BC_DIRICHLET_NEUMANN>(a, g, bc, nb, sh, fs_keep); break;
    case BC_OPEN: band_moments<BC_OPEN>(a, g, bc, nb, sh, fs_keep); break;
    case BC_SETTLING: band_moments<BC_SETTLING>(a, g, bc, nb, sh, fs_keep); break;
    default: band_moments<BC_VELOCITY_INLET>(a, g, bc, nb, sh, fs_keep); break;
    }
    __syncthreads();

    const size_t pstride = 2 * (size_t)NB;
    if (METHOD == IBM_DF) {
        // iblbm/ibm/df.py:93-154, summed over particles as ibm/multi_particle.py:404-421
        const bool incomp = a.c.incompressible != 0;
        for (int l = tid; l < Lb; l += IBM_THREADS) {
            double R, ux, uy;
            {
                double dummy;
                interp2<A>(sh, sh.bro, sh.bro, l, R, dummy);
            }
            interp2<A>(sh, sh.bwx, sh.bwy, l, ux, uy);
            sh.R[l] = R; sh.Lux[l] = ux; sh.Luy[l] = uy;
            double fx, fy;
            if (incomp) { fx = 2.0 * (sh.dvx[l] - ux); fy = 2.0 * (sh.dvy[l] - uy); }
            else { fx = 2.0 * R * (sh.dvx[l] - ux); fy = 2.0 * R * (sh.dvy[l] - uy); }
            sh.Lfx[l] = unit_dt ? fx : fx / dt;
            sh.Lfy[l] = unit_dt ? fy : fy / dt;
        }
        __syncthreads();
        for (int b = tid; b < nb; b += IBM_THREADS) {
            const int u0 = sh.cstart[b], u1 = sh.cstart[b + 1];
            double tx = 0.0, ty = 0.0;
            if (P == 1) {
                spread2(sh, sh.Lfx, sh.Lfy, u0, u1, tx, ty);
                if (a.band_fib_part) { a.band_fib_part[2 * b] = tx; a.band_fib_part[2 * b + 1] = ty; }
                tx = 0.0 + tx;
                ty = 0.0 + ty;
            } else {
                for (int p = 0; p < P; ++p) {
                    double ax = 0.0, ay = 0.0;
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
        double vs[NPT], ftx[NPT], fty[NPT];
#pragma unroll
        for (int jn = 0; jn < NPT; ++jn) {
            const int b = tid + jn * IBM_THREADS;
            vs[jn] = b < nb ? dt / (2.0 * sh.bro[b]) : 0.0;
            ftx[jn] = 0.0;
            fty[jn] = 0.0;
            if (COUPLED && b < nb && a.band_fib_part)
                for (int p = 0; p < P; ++p) {
                    a.band_fib_part[p * pstride + 2 * b] = 0.0;
                    a.band_fib_part[p * pstride + 2 * b + 1] = 0.0;
                }
        }
        const bool own = tid < Lb;  // Lb <= IBM_THREADS (checked on the host)
        const int lo = own ? tid : 0;
        int hb[S];
        double hwx[SW], hwy[SW];
#pragma unroll
        for (int k = 0; k < S; ++k) hb[k] = sh.sidx[lo * S + k];
#pragma unroll
        for (int d = 0; d < SW; ++d) { hwx[d] = sh.wx[lo * 5 + d]; hwy[d] = sh.wy[lo * 5 + d]; }
        const double dvx = sh.dvx[lo], dvy = sh.dvy[lo];
        const int pl = COUPLED ? sh.part[lo] : 0;
        double R = 0.0;
        if (own) {
#pragma unroll
            for (int k = 0; k < S; ++k) R += sh.bro[hb[k]] * (hwx[k / SW] * hwy[k % SW]);
            sh.R[lo] = R;
        }
        const int min_iter = max(1, min(a.mdf_min_iterations, a.mdf_iterations));
        double omega = a.mdf_omega, omega_min = 0.0;
        if (COUPLED) {
            omega = fmin(a.mdf_omega * 0.8, a.mdf_omega_max);
            omega_min = omega * 0.125;
        }
        double prev = INFINITY, last = INFINITY;
        int iter_count = 0, diverged = 0, converged = 0, guard = 0;
        __syncthreads();
        for (int it = 0; it < a.mdf_iterations; ++it) {
            double* wr = sh.wred + (it & 1) * MAXP * NWARP;
            // phase A: interpolate the working velocity, slip residual, force
            double rl = -INFINITY;
            if (own) {
                double ux = 0.0, uy = 0.0;
#pragma unroll
                for (int gi = 0; gi < SW; ++gi) {  // one stencil row (di) at a time, slots in order
                    double vx[SW], vy[SW];
#pragma unroll
                    for (int gj = 0; gj < SW; ++gj) {
                        vx[gj] = sh.bwx[hb[gi * SW + gj]];
                        vy[gj] = sh.bwy[hb[gi * SW + gj]];
                    }
#pragma unroll
                    for (int gj = 0; gj < SW; ++gj) {
                        const double w = hwx[gi] * hwy[gj];
                        ux += vx[gj] * w;
                        uy += vy[gj] * w;
                    }
                }
                sh.Lux[lo] = ux;
                sh.Luy[lo] = uy;
                const double ex = dvx - ux, ey = dvy - uy;
                rl = sqrt(ex * ex + ey * ey);
                double fx, fy;
                if (incomp) { fx = 2.0 * (dvx - ux); fy = 2.0 * (dvy - uy); }
                else { fx = 2.0 * R * (dvx - ux); fy = 2.0 * R * (dvy - uy); }
                sh.Lfx[lo] = unit_dt ? fx : fx / dt;
                sh.Lfy[lo] = unit_dt ? fy : fy / dt;
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
                omega = fmax(omega * 0.5, omega_min);
                if (omega <= omega_min) {
                    diverged = 1;
                    break;
                }
                prev = residual;
                continue;
            }
            // phase B: spread, relax, update the working velocity of the owned nodes
#pragma unroll
            for (int jn = 0; jn < NPT; ++jn) {
                const int b = tid + jn * IBM_THREADS;
                if (b < nb) {
                    const int u0 = sh.cstart[b], u1 = sh.cstart[b + 1];
                    double tx, ty;
                    if (!COUPLED) {
                        double ax, ay;
                        spread2(sh, sh.Lfx, sh.Lfy, u0, u1, ax, ay);
                        tx = ax * omega;
                        ty = ay * omega;
                    } else {
                        tx = 0.0;
                        ty = 0.0;
                        for (int p = 0; p < P; ++p) {
                            double ax = 0.0, ay = 0.0;
                            for (int u = u0; u < u1; ++u) {
                                const int l = sh.ent[u] >> 5;
                                if (sh.part[l] != p) continue;
                                ax += sh.Lfx[l] * sh.entw[u];
                                ay += sh.Lfy[l] * sh.entw[u];
                            }
                            const double fx = ax * omega, fy = ay * omega;
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
                        sh.bwx[b] += 0.5 * tx * dt;
                        sh.bwy[b] += 0.5 * ty * dt;
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
#pragma unroll
        for (int jn = 0; jn < NPT; ++jn) {
            const int b = tid + jn * IBM_THREADS;
            if (b < nb) {
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
            a.stats[3] = guard;
            a.dstats[0] = last;
            a.dstats[1] = omega;
        }
    } else if (METHOD == IBM_DFC) {
        // iblbm/ibm/dfc.py: compute_lambda (126-186) unless cached, interpolate_f
        // (55-95), bounce_back_fi (98-123), spread_delta_f (189-229),
        // compute_dfc_fluid_force (232-253)
        const double La = a.larea[0];
        const bool have = a.dfc_cache_lambda && a.lambda_valid && *a.lambda_valid;
        if (!have) {
            for (int b = tid; b < nb; b += IBM_THREADS) {
                double wt = 0.0;
                for (int u = sh.cstart[b]; u < sh.cstart[b + 1]; ++u) {
                    const int e = sh.ent[u];
                    wt += wgt<A>(sh, e >> 5, e & 31);
                }
                sh.bwx[b] = wt;  // W_total
            }
            __syncthreads();
            for (int l = tid; l < Lb; l += IBM_THREADS) {
                double ws, dummy;
                interp2<A>(sh, sh.bwx, sh.bwx, l, ws, dummy);
                a.lambda[l] = 1.0 / (2.0 * 1.0 * La * ws);
            }
            __syncthreads();
            if (tid == 0 && a.dfc_cache_lambda && a.lambda_valid) *a.lambda_valid = 1;
        }
        const double cs2 = 1.0 / 3.0;
        for (int l = tid; l < Lb; l += IBM_THREADS) {
            double fi[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) fi[q] = 0.0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int b = sh.sidx[l * S + k];
                const double w = wgt<A>(sh, l, k);
#pragma unroll
                for (int q = 0; q < 9; ++q) fi[q] += bfs[9 * (size_t)b + q] * w;
            }
            const double lam = a.lambda[l];
            double sx = 0.0, sy = 0.0;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const double edu = e_dot(q, sh.dvx[l], sh.dvy[l]);
                const double fbb = fi[opp_(q)] + 2.0 * w_(q) * 1.0 * edu / cs2;
                const double dev = fbb - fi[q];
                dfl[9 * (size_t)l + q] = a.correction_scale * lam * dev;
                const double s = -(lam * dev * La);
                sx += s * (double)ex_(q);
                sy += s * (double)ey_(q);
            }
            if (a.dfc_force) {
                a.dfc_force[2 * l] = a.correction_scale * sx;
                a.dfc_force[2 * l + 1] = a.correction_scale * sy;
            }
        }
        __syncthreads();
        for (int b = tid; b < nb; b += IBM_THREADS) {
            double acc[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] = 0.0;
            for (int u = sh.cstart[b]; u < sh.cstart[b + 1]; ++u) {
                const int l = sh.ent[u] >> 5;
                const double w = sh.entw[u];
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

void make_params(const iblbm_case& c, CollParams& cp, BcParams& bc);

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_ibm_smem_bytes(int lb_total, int band_capacity, int delta_type)
{
    const int S = delta_type == 0 ? 25 : 9;
    return (int)make_layout(lb_total, band_capacity, S).total;
}

extern "C" int iblbm_ibm_scratch_doubles(int lb_total, int band_capacity, int n_particles)
{
    (void)n_particles;
    return 9 * band_capacity + 9 * lb_total;
}

extern "C" int iblbm_ibm_scratch_ints(int lb_total, int band_capacity, int delta_type)
{
    (void)lb_total;
    (void)delta_type;
    return band_capacity;
}

extern "C" int iblbm_ibm_list_cache_ints(int lb_total, int band_capacity, int delta_type)
{
    const int S = delta_type == 0 ? 25 : 9;
    return (int)(make_layout(lb_total, band_capacity, S).static_bytes / sizeof(int));
}

// Launch one instantiation; the first launch of each sets its shared-memory limit.
template <void (*K)(const iblbm_ibm_args, BcParams)>
static cudaError_t launch_ibm(const iblbm_ibm_args& a, const BcParams& bc, size_t smem, void* stream)
{
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    K<<<1, IBM_THREADS, smem, (cudaStream_t)stream>>>(a, bc);
    return cudaGetLastError();
}

extern "C" int iblbm_ibm_step_f64(const iblbm_ibm_args* a, void* stream)
{
    if (!a || !a->moff || a->n_particles < 1 || a->n_particles > MAXP || a->lb_total < 1 || !a->fpost_prev ||
        !a->box || !a->map || !a->band_nodes || !a->band_count || !a->scratch || !a->iscratch || !a->stats ||
        !a->dstats || !a->larea || !a->list_cache)
        return IBLBM_E_ARG;
    if (a->delta_type != 0 && a->delta_type != 1) return IBLBM_E_ARG;
    if (a->method != IBM_DF && a->method != IBM_MDF && a->method != IBM_DFC) return IBLBM_E_ARG;
    if ((a->method == IBM_DF || a->method == IBM_MDF) && !a->band_fib) return IBLBM_E_ARG;
    if (a->method == IBM_DFC && (!a->band_df || !a->lambda || a->n_particles != 1)) return IBLBM_E_ARG;
    if (!a->xt_table && (!a->Lx || !a->Ly || !a->dvel)) return IBLBM_E_ARG;
    if (a->xt_table && (!a->Lx_c || !a->Ly_c || !a->step_counter || a->xt_len < 1)) return IBLBM_E_ARG;
    if ((a->c.bc == BC_OPEN || a->c.bc == BC_VELOCITY_INLET) && !a->uring_prev) return IBLBM_E_ARG;
    if (a->band_capacity < 1 || a->band_capacity > MAX_BAND || a->g.nx < 4 || a->g.ny < 4)
        return IBLBM_E_ARG;
    if ((long long)a->lb_total * 32 >= (1LL << 31)) return IBLBM_E_ARG;
    if ((reinterpret_cast<uintptr_t>(a->list_cache) & 15) != 0) return IBLBM_E_ARG;  // bulk-copy source
    const int S = a->delta_type == 0 ? 25 : 9;
    const size_t smem = make_layout(a->lb_total, a->band_capacity, S).total;
    if (smem > 220 * 1024) return IBLBM_E_CAPACITY;
    if (a->method == IBM_MDF && a->lb_total > IBM_THREADS) return IBLBM_E_CAPACITY;
    CollParams cp;
    BcParams bc;
    make_params(a->c, cp, bc);
    const bool coupled = a->method == IBM_MDF && a->mdf_coupled;
    cudaError_t e = cudaErrorInvalidValue;
    if (a->delta_type == 0) {
        if (a->method == IBM_DF) e = launch_ibm<ibm_step_kernel<2, IBM_DF, false>>(*a, bc, smem, stream);
        else if (a->method == IBM_DFC) e = launch_ibm<ibm_step_kernel<2, IBM_DFC, false>>(*a, bc, smem, stream);
        else if (coupled) e = launch_ibm<ibm_step_kernel<2, IBM_MDF, true>>(*a, bc, smem, stream);
        else e = launch_ibm<ibm_step_kernel<2, IBM_MDF, false>>(*a, bc, smem, stream);
    } else {
        if (a->method == IBM_DF) e = launch_ibm<ibm_step_kernel<1, IBM_DF, false>>(*a, bc, smem, stream);
        else if (a->method == IBM_DFC) e = launch_ibm<ibm_step_kernel<1, IBM_DFC, false>>(*a, bc, smem, stream);
        else if (coupled) e = launch_ibm<ibm_step_kernel<1, IBM_MDF, true>>(*a, bc, smem, stream);
        else e = launch_ibm<ibm_step_kernel<1, IBM_MDF, false>>(*a, bc, smem, stream);
    }
    if (e != cudaSuccess) return IBLBM_E_LAUNCH;
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

// ---------------------------------------------------------------------------
// Band step without caller-provided scratch.
//
// Some callers cannot allocate device memory when they call into this library:
// a host framework that owns every device allocation through its own pool and
// hands plugins only the buffers they declared, or a long-running service that
// forbids cudaMalloc after start-up because cudaMalloc can synchronize the
// device and stall its other streams.  For them this entry point takes the
// band kernel's per-launch scratch (the post-streaming populations and
// distribution corrections of the DFC path, and the list-building counters)
// from a fixed array compiled into the library instead of from the caller.
//
// Limits: band_capacity <= 4096 nodes and lb_total <= 1024 markers; larger
// arguments return IBLBM_E_CAPACITY before anything is launched.  The array
// (about 390 KB) lives on every GPU that loads the library until the process
// exits.  All calls share it and it keeps the last call's contents (the kernel
// clears the counters it needs zeroed), so two calls whose kernels overlap on
// the GPU race on it: issue them on one stream, or order them.  The first call
// on each device looks up the array's device address (cudaGetSymbolAddress) with
// that device current; make that first call before any stream capture.  The
// caller still passes every input, output and persistent band array.
// ---------------------------------------------------------------------------
namespace iblbm {
constexpr int NOALLOC_MAX_BAND = 4096;
constexpr int NOALLOC_MAX_MARKERS = 1024;
constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) double g_noalloc_scratch[9 * NOALLOC_MAX_BAND + 9 * NOALLOC_MAX_MARKERS];
static __device__ __align__(256) int g_noalloc_iscratch[NOALLOC_MAX_BAND];
static void* g_noalloc_scratch_ptr[NOALLOC_MAX_DEVICES];
static void* g_noalloc_iscratch_ptr[NOALLOC_MAX_DEVICES];
}  // namespace iblbm

extern "C" int iblbm_ibm_step_f64_noalloc(const iblbm_ibm_args* a, void* stream)
{
    if (!a) return IBLBM_E_ARG;
    if (a->band_capacity > NOALLOC_MAX_BAND || a->lb_total > NOALLOC_MAX_MARKERS) return IBLBM_E_CAPACITY;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return IBLBM_E_LAUNCH;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return IBLBM_E_ARG;
    if (!g_noalloc_scratch_ptr[dev]) {
        void *p = nullptr, *q = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return IBLBM_E_LAUNCH;
        if (cudaGetSymbolAddress(&q, g_noalloc_iscratch) != cudaSuccess) return IBLBM_E_LAUNCH;
        g_noalloc_iscratch_ptr[dev] = q;
        g_noalloc_scratch_ptr[dev] = p;
    }
    iblbm_ibm_args b = *a;
    b.scratch = static_cast<double*>(g_noalloc_scratch_ptr[dev]);
    b.iscratch = static_cast<int*>(g_noalloc_iscratch_ptr[dev]);
    return iblbm_ibm_step_f64(&b, stream);
}
