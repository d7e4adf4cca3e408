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
//     applies the reference's scatter.
//   every step
//     post-streaming populations and moments on the band (the dense kernel's
//     device functions), then DF, MDF (every iteration resident on chip: two
//     barriers per iteration, residual reduced in shared memory, no host round
//     trip), coupled multi-particle MDF, or DFC.
//   exclusion box
//     the band's bounding box dilated by one node is written for the next
//     step: markers move less than one node per step, so the next band lies
//     inside it.  The bulk collide-stream kernel of the next step skips that
//     box and runs concurrently with this kernel; a small box kernel updates
//     the box once this kernel has produced the band forces.
//
// Marker data, band moments and the contribution lists live in shared memory;
// each band node belongs to one thread, which keeps its accumulators in
// registers.  All sums run in the reference's order, so results are
// bit-identical to the reference CPU path (built with -fmad=false).
#include <climits>
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int IBM_THREADS = 512;
constexpr int NPT = 8;     // band nodes per thread: band capacity <= 4096
constexpr int MAXP = 8;    // particles per band kernel
constexpr int NWARP = IBM_THREADS / 32;

enum IbmStatus : int { ST_OK = 0, ST_BAND_CAPACITY = 1, ST_BOX_CAPACITY = 2, ST_MARKERS = 3, ST_TABLE = 4,
                       ST_EXCL = 5 };

template <int A>
struct Sten {
    static constexpr int SW = 2 * A + 1;
    static constexpr int S = SW * SW;
};

__host__ __device__ inline size_t ibm_smem_bytes_t(int Lb, int NB, int S)
{
    size_t s = 0;
    s += sizeof(double) * (size_t)Lb * 17;            // wx[5], wy[5], dvx, dvy, R, Lux, Luy, Lfx, Lfy
    s += sizeof(double) * (size_t)NB * 3;             // band rho, U_work x, U_work y
    s += sizeof(double) * 2 * MAXP * NWARP;           // warp partial maxima
    s += sizeof(int) * (size_t)Lb * (3 + 2 * S);      // ix0, iy0, part, sidx[S], entries[S]
    s += sizeof(int) * ((size_t)NB + 1);              // list starts
    s += sizeof(int) * 64;                            // scan scratch
    return (s + 15) & ~size_t(15);
}

struct Sm {
    double *wx, *wy, *dvx, *dvy, *R, *Lux, *Luy, *Lfx, *Lfy, *bro, *bwx, *bwy, *wred;
    int *ix0, *iy0, *part, *sidx, *cent, *cstart, *ired;
};

template <int S>
__device__ Sm carve(char* base, int Lb, int NB)
{
    Sm s;
    double* d = reinterpret_cast<double*>(base);
    s.wx = d; d += 5 * Lb;
    s.wy = d; d += 5 * Lb;
    s.dvx = d; d += Lb;
    s.dvy = d; d += Lb;
    s.R = d; d += Lb;
    s.Lux = d; d += Lb;
    s.Luy = d; d += Lb;
    s.Lfx = d; d += Lb;
    s.Lfy = d; d += Lb;
    s.bro = d; d += NB;
    s.bwx = d; d += NB;
    s.bwy = d; d += NB;
    s.wred = d; d += 2 * MAXP * NWARP;
    int* p = reinterpret_cast<int*>(d);
    s.ix0 = p; p += Lb;
    s.iy0 = p; p += Lb;
    s.part = p; p += Lb;
    s.sidx = p; p += S * Lb;
    s.cent = p; p += S * Lb;
    s.cstart = p; p += NB + 1;
    s.ired = p;
    return s;
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

template <int BC>
__device__ void band_moments(const iblbm_ibm_args& a, const Geom& g, const BcParams& bc, int nb, const int* nodes,
                             Sm& sh, double* bfs)
{
    const bool incomp = a.c.incompressible != 0;
    for (int b = threadIdx.x; b < nb; b += IBM_THREADS) {
        const int n = nodes[b];
        const int j = n / g.nx, i = n - j * g.nx;
        double f[9];
        fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i, j, f);
        if (bfs) {
#pragma unroll
            for (int q = 0; q < 9; ++q) bfs[9 * (size_t)b + q] = f[q];
        }
        double ro, u0, u1;
        macro_seq(f, incomp, ro, u0, u1);
        sh.bro[b] = ro;
        sh.bwx[b] = u0;
        sh.bwy[b] = u1;
    }
}

template <int A>
__device__ __forceinline__ double wgt(const Sm& sh, int l, int k)
{
    constexpr int SW = Sten<A>::SW;
    return sh.wx[l * 5 + k / SW] * sh.wy[l * 5 + k % SW];
}

template <int A>
__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_step_kernel(const iblbm_ibm_args a, BcParams bc)
{
    constexpr int SW = Sten<A>::SW, S = Sten<A>::S;
    extern __shared__ __align__(16) char smem_raw[];
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int P = a.n_particles, Lb = a.lb_total, NB = a.band_capacity;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    __shared__ int s_nb, s_status, s_box[4], s_step;
    if (tid == 0) {
        s_status = ST_OK;
        s_step = a.step_counter ? *a.step_counter : 0;
        if (a.xt_table && (s_step < 0 || s_step >= a.xt_len)) s_status = ST_TABLE;
    }
    __syncthreads();
    if (s_status != ST_OK) {
        if (tid == 0) a.stats[4] = s_status;
        return;
    }
    Sm sh = carve<S>(smem_raw, Lb, NB);
    const double dx = a.dx, dy = a.dy, dt = a.c.dt;
    double* bfs = a.scratch;                       // 9 * NB post-streaming populations (DFC)
    double* dfl = a.scratch + 9 * (size_t)NB;      // 9 * Lb distribution corrections (DFC)
    int* cfill = a.iscratch;                       // NB
    int* nodes = a.band_nodes;

    // ---- markers of this step ------------------------------------------------
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
        int p = 0;
        while (p + 1 < P && l >= a.moff[p + 1]) ++p;
        sh.part[l] = p;
        // iblbm/ibm/df.py:94-114: nearest node and separable weights
        const double fx = floor(x / dx + 0.5), fy = floor(y / dy + 0.5);
        const long long ix0 = (long long)fmin(fmax(fx, -1.0e9), 1.0e9);
        const long long iy0 = (long long)fmin(fmax(fy, -1.0e9), 1.0e9);
        sh.ix0[l] = (int)ix0;
        sh.iy0[l] = (int)iy0;
#pragma unroll
        for (int d = -A; d <= A; ++d) {
            sh.wx[l * 5 + d + A] = phi(A == 2 ? 0 : 1, (x - (double)(ix0 + d) * dx) / dx);
            sh.wy[l * 5 + d + A] = phi(A == 2 ? 0 : 1, (y - (double)(iy0 + d) * dy) / dy);
        }
    }
    __syncthreads();

    auto node_of = [&](int l, int k) -> long long {
        const int ei = min(max(sh.ix0[l] + k / SW - A, 0), g.nx - 1);
        const int ej = min(max(sh.iy0[l] + k % SW - A, 0), g.ny - 1);
        return (long long)ej * g.nx + ei;
    };

    int nb;
    if (a.rebuild || a.xt_table) {
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
        for (int b = tid; b < nprev; b += IBM_THREADS) a.map[nodes[b]] = -1;  // clear the previous band
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
                    nodes[idx] = (int)n;
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
            sh.cent[sh.cstart[b] + atomicAdd(&cfill[b], 1)] = (l << 5) | k;
        }
        __syncthreads();
        // order each list by (k, l): the reference's scatter order
        for (int b = tid; b < nb; b += IBM_THREADS) {
            const int s0 = sh.cstart[b], s1 = sh.cstart[b + 1];
            for (int u = s0 + 1; u < s1; ++u) {
                const int v = sh.cent[u];
                const int kv = v & 31, lv = v >> 5;
                int w = u - 1;
                while (w >= s0) {
                    const int c = sh.cent[w];
                    const int kc = c & 31, lc = c >> 5;
                    if (kc < kv || (kc == kv && lc < lv)) break;
                    sh.cent[w + 1] = c;
                    --w;
                }
                sh.cent[w + 1] = v;
            }
        }
        __syncthreads();
        for (int u = tid; u < S * Lb; u += IBM_THREADS) a.list_cache[u] = sh.cent[u];
        for (int b = tid; b <= nb; b += IBM_THREADS) a.list_cache[S * Lb + b] = sh.cstart[b];
        if (tid == 0) s_nb = nb;
        __syncthreads();
    } else {
        if (tid == 0) {
            s_nb = *a.band_count;
            s_box[0] = a.box[0];
            s_box[1] = a.box[1];
            s_box[2] = a.box[0] + a.box[2] - 1;
            s_box[3] = a.box[1] + a.box[3] - 1;
        }
        __syncthreads();
        nb = s_nb;
        for (int e = tid; e < S * Lb; e += IBM_THREADS) {
            const int l = e % Lb, k = e / Lb;
            sh.sidx[l * S + k] = a.map[node_of(l, k)];
        }
        for (int u = tid; u < S * Lb; u += IBM_THREADS) sh.cent[u] = a.list_cache[u];
        for (int b = tid; b <= nb; b += IBM_THREADS) sh.cstart[b] = a.list_cache[S * Lb + b];
        __syncthreads();
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
    double* fs_keep = (a.method == IBM_DFC) ? bfs : nullptr;
    switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN: band_moments<BC_DIRICHLET_NEUMANN>(a, g, bc, nb, nodes, sh, fs_keep); break;
    case BC_OPEN: band_moments<BC_OPEN>(a, g, bc, nb, nodes, sh, fs_keep); break;
    case BC_SETTLING: band_moments<BC_SETTLING>(a, g, bc, nb, nodes, sh, fs_keep); break;
    default: band_moments<BC_VELOCITY_INLET>(a, g, bc, nb, nodes, sh, fs_keep); break;
    }
    __syncthreads();

    const size_t pstride = 2 * (size_t)NB;
    if (a.method == IBM_DF) {
        // iblbm/ibm/df.py:93-154, summed over particles as ibm/multi_particle.py:404-421
        const bool incomp = a.c.incompressible != 0;
        for (int l = tid; l < Lb; l += IBM_THREADS) {
            double R = 0.0, ux = 0.0, uy = 0.0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int b = sh.sidx[l * S + k];
                const double w = wgt<A>(sh, l, k);
                R += sh.bro[b] * w;
                ux += sh.bwx[b] * w;
                uy += sh.bwy[b] * w;
            }
            sh.R[l] = R; sh.Lux[l] = ux; sh.Luy[l] = uy;
            if (incomp) {
                sh.Lfx[l] = 2.0 * (sh.dvx[l] - ux) / dt;
                sh.Lfy[l] = 2.0 * (sh.dvy[l] - uy) / dt;
            } else {
                sh.Lfx[l] = 2.0 * R * (sh.dvx[l] - ux) / dt;
                sh.Lfy[l] = 2.0 * R * (sh.dvy[l] - uy) / dt;
            }
        }
        __syncthreads();
        for (int b = tid; b < nb; b += IBM_THREADS) {
            double tx = 0.0, ty = 0.0;
            for (int p = 0; p < P; ++p) {
                const double La = a.larea[p];
                double ax = 0.0, ay = 0.0;
                for (int u = sh.cstart[b]; u < sh.cstart[b + 1]; ++u) {
                    const int e = sh.cent[u], l = e >> 5, k = e & 31;
                    if (sh.part[l] != p) continue;
                    const double w = wgt<A>(sh, l, k) * La;
                    ax += sh.Lfx[l] * w;
                    ay += sh.Lfy[l] * w;
                }
                if (a.band_fib_part) {
                    a.band_fib_part[p * pstride + 2 * b] = ax;
                    a.band_fib_part[p * pstride + 2 * b + 1] = ay;
                }
                tx += ax;
                ty += ay;
            }
            a.band_fib[2 * b] = tx;
            a.band_fib[2 * b + 1] = ty;
        }
    } else if (a.method == IBM_MDF) {
        // iblbm/ibm/mdf.py:61-229 (one body) and iblbm/ibm/multi_particle.py:62-316 (coupled)
        const bool coupled = a.mdf_coupled != 0;
        const bool incomp = coupled && a.c.incompressible != 0;  // mdf.py always uses the compressible law
        double vs[NPT], ftx[NPT], fty[NPT];
#pragma unroll
        for (int jn = 0; jn < NPT; ++jn) {
            const int b = tid + jn * IBM_THREADS;
            vs[jn] = b < nb ? dt / (2.0 * sh.bro[b]) : 0.0;
            ftx[jn] = 0.0;
            fty[jn] = 0.0;
            if (b < nb && coupled && a.band_fib_part)
                for (int p = 0; p < P; ++p) {
                    a.band_fib_part[p * pstride + 2 * b] = 0.0;
                    a.band_fib_part[p * pstride + 2 * b + 1] = 0.0;
                }
        }
        for (int l = tid; l < Lb; l += IBM_THREADS) {
            double R = 0.0;
#pragma unroll
            for (int k = 0; k < S; ++k) R += sh.bro[sh.sidx[l * S + k]] * wgt<A>(sh, l, k);
            sh.R[l] = R;
        }
        const int min_iter = max(1, min(a.mdf_min_iterations, a.mdf_iterations));
        double omega = a.mdf_omega, omega_min = 0.0;
        if (coupled) {
            omega = fmin(a.mdf_omega * 0.8, a.mdf_omega_max);
            omega_min = omega * 0.125;
        }
        double prev = INFINITY, last = INFINITY;
        int iter_count = 0, diverged = 0, converged = 0, guard = 0;
        __syncthreads();
        for (int it = 0; it < a.mdf_iterations; ++it) {
            double* wr = sh.wred + (it & 1) * MAXP * NWARP;
            // phase A: interpolate the working velocity, slip residual, force
            double rl[MAXP];
#pragma unroll
            for (int p = 0; p < MAXP; ++p) rl[p] = -INFINITY;
            for (int l = tid; l < Lb; l += IBM_THREADS) {
                double ux = 0.0, uy = 0.0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    const int b = sh.sidx[l * S + k];
                    const double w = wgt<A>(sh, l, k);
                    ux += sh.bwx[b] * w;
                    uy += sh.bwy[b] * w;
                }
                sh.Lux[l] = ux;
                sh.Luy[l] = uy;
                const double vx = sh.dvx[l] - ux, vy = sh.dvy[l] - uy;
                const double r = sqrt(vx * vx + vy * vy);
                const int pl = coupled ? sh.part[l] : 0;
#pragma unroll
                for (int p = 0; p < MAXP; ++p)
                    if (p == pl) rl[p] = nanmax(rl[p], r);
                if (incomp) {
                    sh.Lfx[l] = 2.0 * (sh.dvx[l] - ux) / dt;
                    sh.Lfy[l] = 2.0 * (sh.dvy[l] - uy) / dt;
                } else {
                    sh.Lfx[l] = 2.0 * sh.R[l] * (sh.dvx[l] - ux) / dt;
                    sh.Lfy[l] = 2.0 * sh.R[l] * (sh.dvy[l] - uy) / dt;
                }
            }
            const int np = coupled ? P : 1;
#pragma unroll
            for (int p = 0; p < MAXP; ++p) {
                if (p >= np) break;
                const double v = warp_nanmax(rl[p]);
                if (lane == 0) wr[p * NWARP + wid] = v;
            }
            __syncthreads();  // (a)
            double residual;
            if (!coupled) {
                residual = -INFINITY;
                for (int w = 0; w < NWARP; ++w) residual = nanmax(residual, wr[w]);
            } else {
                residual = 0.0;  // Python max over the particles' numpy maxima, from 0.0
                for (int p = 0; p < P; ++p) {
                    double rp = -INFINITY;
                    for (int w = 0; w < NWARP; ++w) rp = nanmax(rp, wr[p * NWARP + w]);
                    if (rp > residual) residual = rp;
                }
            }
            last = residual;
            if (!coupled) {
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
                if (b >= nb) break;
                const int u0 = sh.cstart[b], u1 = sh.cstart[b + 1];
                double tx = 0.0, ty = 0.0;
                for (int p = 0; p < P; ++p) {
                    const double La = a.larea[p];
                    double ax = 0.0, ay = 0.0;
                    for (int u = u0; u < u1; ++u) {
                        const int e = sh.cent[u], l = e >> 5, k = e & 31;
                        if (P > 1 && sh.part[l] != p) continue;
                        const double w = wgt<A>(sh, l, k) * La;
                        ax += sh.Lfx[l] * w;
                        ay += sh.Lfy[l] * w;
                    }
                    const double fx = ax * omega, fy = ay * omega;
                    if (coupled && a.band_fib_part) {
                        a.band_fib_part[p * pstride + 2 * b] += fx;
                        a.band_fib_part[p * pstride + 2 * b + 1] += fy;
                    }
                    tx += fx;
                    ty += fy;
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
            __syncthreads();  // (b)
            prev = residual;
            if (coupled) iter_count += 1;
            else iter_count = it + 1;
            if ((it + 1) >= min_iter && residual < a.mdf_tol) {
                converged = 1;
                break;
            }
        }
#pragma unroll
        for (int jn = 0; jn < NPT; ++jn) {
            const int b = tid + jn * IBM_THREADS;
            if (b >= nb) break;
            a.band_fib[2 * b] = ftx[jn];
            a.band_fib[2 * b + 1] = fty[jn];
            if (!coupled && a.band_fib_part) {
                a.band_fib_part[2 * b] = ftx[jn];
                a.band_fib_part[2 * b + 1] = fty[jn];
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
    } else if (a.method == IBM_DFC) {
        // iblbm/ibm/dfc.py: compute_lambda (126-186) unless cached, interpolate_f
        // (55-95), bounce_back_fi (98-123), spread_delta_f (189-229),
        // compute_dfc_fluid_force (232-253)
        const double La = a.larea[0];
        const bool have = a.dfc_cache_lambda && a.lambda_valid && *a.lambda_valid;
        if (!have) {
            for (int b = tid; b < nb; b += IBM_THREADS) {
                double wt = 0.0;
                for (int u = sh.cstart[b]; u < sh.cstart[b + 1]; ++u) {
                    const int e = sh.cent[u];
                    wt += wgt<A>(sh, e >> 5, e & 31);
                }
                sh.bwx[b] = wt;  // W_total
            }
            __syncthreads();
            for (int l = tid; l < Lb; l += IBM_THREADS) {
                double ws = 0.0;
#pragma unroll
                for (int k = 0; k < S; ++k) ws += sh.bwx[sh.sidx[l * S + k]] * wgt<A>(sh, l, k);
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
                const int e = sh.cent[u], l = e >> 5, k = e & 31;
                const double w = wgt<A>(sh, l, k) * La;
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
    return (int)ibm_smem_bytes_t(lb_total, band_capacity, S);
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
    return S * lb_total + band_capacity + 1;
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
    if (a->band_capacity < 1 || a->band_capacity > NPT * IBM_THREADS || a->g.nx < 4 || a->g.ny < 4)
        return IBLBM_E_ARG;
    if ((long long)a->lb_total * 32 >= (1LL << 31)) return IBLBM_E_ARG;
    const int S = a->delta_type == 0 ? 25 : 9;
    const size_t smem = ibm_smem_bytes_t(a->lb_total, a->band_capacity, S);
    if (smem > 220 * 1024) return IBLBM_E_CAPACITY;
    static int configured = 0;
    if (!configured) {
        if (cudaFuncSetAttribute(ibm_step_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024) !=
                cudaSuccess ||
            cudaFuncSetAttribute(ibm_step_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024) !=
                cudaSuccess)
            return IBLBM_E_LAUNCH;
        configured = 1;
    }
    CollParams cp;
    BcParams bc;
    make_params(a->c, cp, bc);
    if (a->delta_type == 0)
        ibm_step_kernel<2><<<1, IBM_THREADS, smem, (cudaStream_t)stream>>>(*a, bc);
    else
        ibm_step_kernel<1><<<1, IBM_THREADS, smem, (cudaStream_t)stream>>>(*a, bc);
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
