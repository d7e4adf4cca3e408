// ibm_f64.cu — immersed-boundary marker loop on the band, FP64.
//
// The band is the set of lattice nodes under the marker stencils (a few hundred
// to a few thousand nodes).  One CTA of 1024 threads owns it for the whole step:
//
//   rebuild (fixed bodies: once; moving bodies: every step)
//     markers -> nearest node ix0 = floor(x/dx + 0.5), separable weights
//     wx[5], wy[5]; bounding box; band compaction in row-major (= lattice
//     index) order; per-node contribution lists (CSR) sorted by the
//     reference's scatter order e = k*Lb + l (stencil slot k = (di outer,
//     dj inner), then marker l), which is the order numpy's add.at applies.
//   every step
//     post-streaming populations and moments on the band (same device
//     functions as the dense kernel), then DF, MDF (all iterations resident,
//     residual reduced on chip, no host round trip), coupled multi-particle
//     MDF, or DFC.
//
// Marker arrays live in shared memory; band arrays in global scratch (they are
// a few tens of KB and stay in L1/L2).  Sums run in the reference's order, so
// results are bit-identical to the reference CPU path (-fmad=false).
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int IBM_THREADS = 1024;
constexpr int MAX_S = 25;  // (2a+1)^2 for the Peskin 4-point kernel

enum IbmStatus : int { ST_OK = 0, ST_BAND_CAPACITY = 1, ST_BOX_CAPACITY = 2, ST_MARKERS = 3, ST_TABLE = 4 };

struct IbmShared {
    int *ix0, *iy0, *sidx, *part;
    double *wx, *wy, *dvx, *dvy, *R, *Lux, *Luy, *Lfx, *Lfy;
    double* red;  // 32 doubles
    int* ired;    // 64 ints
};

__device__ __forceinline__ size_t align8(size_t x) { return (x + 7) & ~size_t(7); }

__host__ __device__ inline size_t ibm_smem_bytes(int Lb)
{
    size_t s = 0;
    s += sizeof(double) * (size_t)Lb * (5 + 5 + 7);
    s += sizeof(double) * 32;
    s += sizeof(int) * (size_t)Lb * (2 + MAX_S + 1);
    s += sizeof(int) * 64;
    return (s + 15) & ~size_t(15);
}

__device__ IbmShared carve(char* base, int Lb)
{
    IbmShared s;
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
    s.red = d; d += 32;
    int* p = reinterpret_cast<int*>(d);
    s.ix0 = p; p += Lb;
    s.iy0 = p; p += Lb;
    s.sidx = p; p += MAX_S * Lb;
    s.part = p; p += Lb;
    s.ired = p;
    return s;
}

// Block-wide max with NaN propagation (numpy max semantics).  All threads
// receive the result.
__device__ double block_max_nan(double v, double* red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = (u > v || u != u) ? u : v;
    }
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double x = (lane < (blockDim.x >> 5)) ? red[lane] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_xor_sync(0xffffffffu, x, o);
            x = (u > x || u != u) ? u : x;
        }
        if (lane == 0) red[0] = x;
    }
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

// Block-wide exclusive scan of one int per thread; returns the prefix and
// writes the total to *total.
__device__ int block_exscan(int v, int* ired, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
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
        int y = lane < nw ? ired[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += u;
        }
        if (lane < nw) ired[32 + lane] = y;
    }
    __syncthreads();
    const int base = wid > 0 ? ired[32 + wid - 1] : 0;
    *total = ired[32 + nw - 1];
    __syncthreads();
    return base + x - v;
}

template <int BC>
__device__ void band_moments(const iblbm_ibm_args& a, const Geom& g, const BcParams& bc, int nb, const int* nodes,
                             double* bro, double* bu0, double* bu1, double* bfs)
{
    const bool incomp = a.c.incompressible != 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int n = nodes[b];
        const int j = n / g.nx, i = n - j * g.nx;
        double f[9];
        fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i, j, f);
        if (bfs) {
#pragma unroll
            for (int q = 0; q < 9; ++q) bfs[9 * b + q] = f[q];
        }
        double ro, u0, u1;
        macro_seq(f, incomp, ro, u0, u1);
        bro[b] = ro;
        bu0[b] = u0;
        bu1[b] = u1;
    }
}

void make_params(const iblbm_case& c, CollParams& cp, BcParams& bc);

__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_step_kernel(const iblbm_ibm_args a, BcParams bc)
{
    extern __shared__ __align__(16) char smem_raw[];
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const int P = a.n_particles;
    __shared__ int s_lb, s_nb, s_status, s_box[4], s_step;
    if (threadIdx.x == 0) {
        s_lb = a.lb_total;
        s_status = ST_OK;
        s_step = a.step_counter ? *a.step_counter : 0;
        if (a.xt_table && (s_step < 0 || s_step >= a.xt_len)) s_status = ST_TABLE;
    }
    __syncthreads();
    if (s_status != ST_OK) {
        if (threadIdx.x == 0) a.stats[4] = s_status;
        return;
    }
    const int Lb = s_lb;
    IbmShared sh = carve(smem_raw, Lb);
    const int A = (a.delta_type == 0) ? 2 : 1;
    const int SW = 2 * A + 1, S = SW * SW;
    const double dx = a.dx, dy = a.dy, dt = a.c.dt;

    // global scratch carve (matches iblbm_ibm_scratch_doubles / _ints)
    const int B = a.band_capacity;
    double* bro = a.scratch;
    double* bu0 = bro + B;
    double* bu1 = bu0 + B;
    double* bvs = bu1 + B;
    double* bwx = bvs + B;       // U_work x (MDF) / W_total (DFC)
    double* bwy = bwx + B;       // U_work y (MDF)
    double* bfs = bwy + B;       // 9 * B post-streaming populations (DFC)
    double* dfl = bfs + 9 * (size_t)B;  // 9 * Lb distribution corrections per marker (DFC)
    int* cstart = a.iscratch;     // B + 1
    int* cfill = cstart + B + 1;  // B
    int* centry = cfill + B;      // Lb * 25
    int* nodes = a.band_nodes;

    // ---- markers for this step -------------------------------------------
    for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
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
        const long long ix0 = (long long)floor(x / dx + 0.5);
        const long long iy0 = (long long)floor(y / dy + 0.5);
        sh.ix0[l] = (int)ix0;
        sh.iy0[l] = (int)iy0;
        for (int d = -A; d <= A; ++d) {
            sh.wx[l * 5 + d + A] = phi(a.delta_type, (x - (double)(ix0 + d) * dx) / dx);
            sh.wy[l * 5 + d + A] = phi(a.delta_type, (y - (double)(iy0 + d) * dy) / dy);
        }
    }
    __syncthreads();

    int nb;
    if (a.rebuild || a.xt_table) {
        // ---- band rebuild ----------------------------------------------------
        if (threadIdx.x == 0) { s_box[0] = INT_MAX; s_box[1] = INT_MAX; s_box[2] = INT_MIN; s_box[3] = INT_MIN; }
        __syncthreads();
        for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
            const int x0 = min(max(sh.ix0[l] - A, 0), g.nx - 1), x1 = min(max(sh.ix0[l] + A, 0), g.nx - 1);
            const int y0 = min(max(sh.iy0[l] - A, 0), g.ny - 1), y1 = min(max(sh.iy0[l] + A, 0), g.ny - 1);
            atomicMin(&s_box[0], x0);
            atomicMin(&s_box[1], y0);
            atomicMax(&s_box[2], x1);
            atomicMax(&s_box[3], y1);
        }
        // clear the previous band's map entries
        const int nprev = *a.band_count;
        for (int b = threadIdx.x; b < nprev; b += blockDim.x) a.map[nodes[b]] = -1;
        __syncthreads();
        const int bx0 = s_box[0], by0 = s_box[1], bw = s_box[2] - s_box[0] + 1, bh = s_box[3] - s_box[1] + 1;
        if ((long long)bw * bh > (long long)a.box_capacity) {
            if (threadIdx.x == 0) s_status = ST_BOX_CAPACITY;
        }
        // mark stencil nodes
        for (int e = threadIdx.x; e < S * Lb; e += blockDim.x) {
            const int l = e % Lb, k = e / Lb;
            const int di = k / SW - A, dj = k % SW - A;
            const int ei = min(max(sh.ix0[l] + di, 0), g.nx - 1), ej = min(max(sh.iy0[l] + dj, 0), g.ny - 1);
            a.map[(long long)ej * g.nx + ei] = -2;
        }
        __syncthreads();
        // compaction over the box in row-major order
        const int cells = bw * bh;
        const int chunk = (cells + blockDim.x - 1) / blockDim.x;
        const int c0 = threadIdx.x * chunk, c1 = min(c0 + chunk, cells);
        int cnt = 0;
        for (int c = c0; c < c1; ++c) {
            const int n = (by0 + c / bw) * g.nx + bx0 + c % bw;
            cnt += (a.map[n] == -2);
        }
        int total;
        int idx = block_exscan(cnt, sh.ired, &total);
        if (total > B) {
            if (threadIdx.x == 0) s_status = ST_BAND_CAPACITY;
            __syncthreads();
        } else {
            for (int c = c0; c < c1; ++c) {
                const int n = (by0 + c / bw) * g.nx + bx0 + c % bw;
                if (a.map[n] == -2) {
                    a.map[n] = idx;
                    nodes[idx] = n;
                    ++idx;
                }
            }
        }
        __syncthreads();
        if (s_status != ST_OK) {
            if (threadIdx.x == 0) {
                a.stats[4] = s_status;
                *a.band_count = 0;
                a.box[0] = 0; a.box[1] = 0; a.box[2] = 0; a.box[3] = 0;
            }
            return;
        }
        nb = total;
        if (threadIdx.x == 0) {
            *a.band_count = nb;
            a.box[0] = bx0; a.box[1] = by0; a.box[2] = bw; a.box[3] = bh;
            s_nb = nb;
        }
        // stencil slot -> band index; contribution counts
        for (int b = threadIdx.x; b <= nb; b += blockDim.x) { cstart[b] = 0; if (b < nb) cfill[b] = 0; }
        __syncthreads();
        for (int e = threadIdx.x; e < S * Lb; e += blockDim.x) {
            const int l = e % Lb, k = e / Lb;
            const int di = k / SW - A, dj = k % SW - A;
            const int ei = min(max(sh.ix0[l] + di, 0), g.nx - 1), ej = min(max(sh.iy0[l] + dj, 0), g.ny - 1);
            const int b = a.map[(long long)ej * g.nx + ei];
            sh.sidx[l * MAX_S + k] = b;
            atomicAdd(&cfill[b], 1);
        }
        __syncthreads();
        // exclusive scan of counts -> cstart
        {
            const int ch = (nb + blockDim.x - 1) / blockDim.x;
            const int b0 = threadIdx.x * ch, b1 = min(b0 + ch, nb);
            int c = 0;
            for (int b = b0; b < b1; ++b) c += cfill[b];
            int tot;
            int base = block_exscan(c, sh.ired, &tot);
            for (int b = b0; b < b1; ++b) { cstart[b] = base; base += cfill[b]; cfill[b] = 0; }
            if (threadIdx.x == 0) cstart[nb] = tot;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < S * Lb; e += blockDim.x) {
            const int l = e % Lb, k = e / Lb;
            const int b = sh.sidx[l * MAX_S + k];
            const int pos = cstart[b] + atomicAdd(&cfill[b], 1);
            centry[pos] = e;
        }
        __syncthreads();
        // sort each node's list by e (insertion sort; lists are short)
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            const int s0 = cstart[b], s1 = cstart[b + 1];
            for (int u = s0 + 1; u < s1; ++u) {
                const int v = centry[u];
                int w = u - 1;
                while (w >= s0 && centry[w] > v) { centry[w + 1] = centry[w]; --w; }
                centry[w + 1] = v;
            }
        }
        __syncthreads();
    } else {
        if (threadIdx.x == 0) s_nb = *a.band_count;
        __syncthreads();
        nb = s_nb;
        for (int e = threadIdx.x; e < S * Lb; e += blockDim.x) {
            const int l = e % Lb, k = e / Lb;
            const int di = k / SW - A, dj = k % SW - A;
            const int ei = min(max(sh.ix0[l] + di, 0), g.nx - 1), ej = min(max(sh.iy0[l] + dj, 0), g.ny - 1);
            sh.sidx[l * MAX_S + k] = a.map[(long long)ej * g.nx + ei];
        }
        __syncthreads();
    }

    // ---- post-streaming populations and moments on the band ----------------
    double* fs_keep = (a.method == IBM_DFC) ? bfs : nullptr;
    switch (a.c.bc) {
    case BC_DIRICHLET_NEUMANN: band_moments<BC_DIRICHLET_NEUMANN>(a, g, bc, nb, nodes, bro, bu0, bu1, fs_keep); break;
    case BC_OPEN: band_moments<BC_OPEN>(a, g, bc, nb, nodes, bro, bu0, bu1, fs_keep); break;
    case BC_SETTLING: band_moments<BC_SETTLING>(a, g, bc, nb, nodes, bro, bu0, bu1, fs_keep); break;
    default: band_moments<BC_VELOCITY_INLET>(a, g, bc, nb, nodes, bro, bu0, bu1, fs_keep); break;
    }
    __syncthreads();

    auto wgt = [&](int l, int k) -> double { return sh.wx[l * 5 + k / SW] * sh.wy[l * 5 + k % SW]; };

    if (a.method == IBM_DF) {
        // iblbm/ibm/df.py:93-154 (per particle: multi_particle_df sums them)
        const bool incomp = a.c.incompressible != 0;
        for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
            double R = 0.0, ux = 0.0, uy = 0.0;
            for (int k = 0; k < S; ++k) {
                const int b = sh.sidx[l * MAX_S + k];
                const double w = wgt(l, k);
                R += bro[b] * w;
                ux += bu0[b] * w;
                uy += bu1[b] * w;
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
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            double tx = 0.0, ty = 0.0;
            for (int p = 0; p < P; ++p) {
                const double La = a.larea[p];
                double ax = 0.0, ay = 0.0;
                for (int u = cstart[b]; u < cstart[b + 1]; ++u) {
                    const int e = centry[u], l = e % Lb, k = e / Lb;
                    if (sh.part[l] != p) continue;
                    const double w = wgt(l, k) * La;
                    ax += sh.Lfx[l] * w;
                    ay += sh.Lfy[l] * w;
                }
                if (a.band_fib_part) {
                    a.band_fib_part[2 * ((size_t)p * B + b)] = ax;
                    a.band_fib_part[2 * ((size_t)p * B + b) + 1] = ay;
                }
                tx += ax;
                ty += ay;
            }
            a.band_fib[2 * b] = tx;
            a.band_fib[2 * b + 1] = ty;
        }
    } else if (a.method == IBM_MDF) {
        // iblbm/ibm/mdf.py:61-229 (P == 1 or not coupled) and
        // iblbm/ibm/multi_particle.py:62-316 (coupled, P >= 2)
        const bool coupled = a.mdf_coupled != 0;
        const bool incomp = coupled && a.c.incompressible != 0;  // mdf.py always uses the compressible law
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            bvs[b] = dt / (2.0 * bro[b]);
            bwx[b] = bu0[b];
            bwy[b] = bu1[b];
            a.band_fib[2 * b] = 0.0;
            a.band_fib[2 * b + 1] = 0.0;
            if (a.band_fib_part)
                for (int p = 0; p < P; ++p) {
                    a.band_fib_part[2 * ((size_t)p * B + b)] = 0.0;
                    a.band_fib_part[2 * ((size_t)p * B + b) + 1] = 0.0;
                }
        }
        for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
            double R = 0.0;
            for (int k = 0; k < S; ++k) R += bro[sh.sidx[l * MAX_S + k]] * wgt(l, k);
            sh.R[l] = R;
        }
        int min_iter = min(a.mdf_min_iterations, a.mdf_iterations);
        min_iter = max(1, min_iter);
        double omega = a.mdf_omega;
        double omega_min = 0.0;
        if (coupled) {
            omega = fmin(a.mdf_omega * 0.8, a.mdf_omega_max);
            omega_min = omega * 0.125;
        }
        double prev = INFINITY, last = INFINITY;
        int iter_count = 0, diverged = 0, converged = 0, guard = 0;
        __syncthreads();
        for (int it = 0; it < a.mdf_iterations; ++it) {
            // interpolation of the working velocity and slip residual
            double rloc = -INFINITY;
            for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
                double ux = 0.0, uy = 0.0;
                for (int k = 0; k < S; ++k) {
                    const int b = sh.sidx[l * MAX_S + k];
                    const double w = wgt(l, k);
                    ux += bwx[b] * w;
                    uy += bwy[b] * w;
                }
                sh.Lux[l] = ux;
                sh.Luy[l] = uy;
                const double vx = sh.dvx[l] - ux, vy = sh.dvy[l] - uy;
                const double r = sqrt(vx * vx + vy * vy);
                if (!coupled) rloc = (r > rloc || r != r) ? r : rloc;
                if (incomp) {
                    sh.Lfx[l] = 2.0 * (sh.dvx[l] - ux) / dt;
                    sh.Lfy[l] = 2.0 * (sh.dvy[l] - uy) / dt;
                } else {
                    sh.Lfx[l] = 2.0 * sh.R[l] * (sh.dvx[l] - ux) / dt;
                    sh.Lfy[l] = 2.0 * sh.R[l] * (sh.dvy[l] - uy) / dt;
                }
            }
            double residual;
            if (!coupled) {
                residual = block_max_nan(rloc, sh.red);
            } else {
                // per-particle numpy max, folded with Python's max starting at 0.0
                __syncthreads();
                residual = 0.0;
                for (int p = 0; p < P; ++p) {
                    double rp = -INFINITY;
                    for (int l = a.moff[p] + threadIdx.x; l < a.moff[p + 1]; l += blockDim.x) {
                        const double vx = sh.dvx[l] - sh.Lux[l], vy = sh.dvy[l] - sh.Luy[l];
                        const double r = sqrt(vx * vx + vy * vy);
                        rp = (r > rp || r != r) ? r : rp;
                    }
                    rp = block_max_nan(rp, sh.red);
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
            // spread, relax and update the working velocity (band nodes)
            for (int b = threadIdx.x; b < nb; b += blockDim.x) {
                double tx = 0.0, ty = 0.0;
                for (int p = 0; p < P; ++p) {
                    const double La = a.larea[p];
                    double ax = 0.0, ay = 0.0;
                    for (int u = cstart[b]; u < cstart[b + 1]; ++u) {
                        const int e = centry[u], l = e % Lb, k = e / Lb;
                        if (sh.part[l] != p) continue;
                        const double w = wgt(l, k) * La;
                        ax += sh.Lfx[l] * w;
                        ay += sh.Lfy[l] * w;
                    }
                    const double fx = ax * omega, fy = ay * omega;
                    if (coupled && a.band_fib_part) {
                        a.band_fib_part[2 * ((size_t)p * B + b)] += fx;
                        a.band_fib_part[2 * ((size_t)p * B + b) + 1] += fy;
                    }
                    tx += fx;
                    ty += fy;
                }
                a.band_fib[2 * b] += tx;
                a.band_fib[2 * b + 1] += ty;
                if (incomp) {
                    bwx[b] += 0.5 * tx * dt;
                    bwy[b] += 0.5 * ty * dt;
                } else {
                    bwx[b] += tx * bvs[b];
                    bwy[b] += ty * bvs[b];
                }
            }
            __syncthreads();
            prev = residual;
            if (coupled) iter_count += 1;
            else iter_count = it + 1;
            if ((it + 1) >= min_iter && residual < a.mdf_tol) {
                converged = 1;
                break;
            }
        }
        if (!coupled && a.band_fib_part) {
            __syncthreads();
            for (int b = threadIdx.x; b < nb; b += blockDim.x) {
                a.band_fib_part[2 * (size_t)b] = a.band_fib[2 * b];
                a.band_fib_part[2 * (size_t)b + 1] = a.band_fib[2 * b + 1];
            }
        }
        if (threadIdx.x == 0) {
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
            for (int b = threadIdx.x; b < nb; b += blockDim.x) {
                double wt = 0.0;
                for (int u = cstart[b]; u < cstart[b + 1]; ++u) {
                    const int e = centry[u], l = e % Lb, k = e / Lb;
                    wt += wgt(l, k);
                }
                bwx[b] = wt;
            }
            __syncthreads();
            for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
                double ws = 0.0;
                for (int k = 0; k < S; ++k) ws += bwx[sh.sidx[l * MAX_S + k]] * wgt(l, k);
                a.lambda[l] = 1.0 / (2.0 * 1.0 * La * ws);
            }
            __syncthreads();
            if (threadIdx.x == 0 && a.dfc_cache_lambda && a.lambda_valid) *a.lambda_valid = 1;
        }
        const double cs2 = 1.0 / 3.0;
        for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
            double fi[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) fi[q] = 0.0;
            for (int k = 0; k < S; ++k) {
                const int b = sh.sidx[l * MAX_S + k];
                const double w = wgt(l, k);
#pragma unroll
                for (int q = 0; q < 9; ++q) fi[q] += bfs[9 * b + q] * w;
            }
            const double lam = a.lambda[l];
            double sx = 0.0, sy = 0.0;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const double edu = e_dot(q, sh.dvx[l], sh.dvy[l]);
                const double fbb = fi[opp_(q)] + 2.0 * w_(q) * 1.0 * edu / cs2;
                const double dev = fbb - fi[q];
                dfl[9 * l + q] = a.correction_scale * lam * dev;
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
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            double acc[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] = 0.0;
            for (int u = cstart[b]; u < cstart[b + 1]; ++u) {
                const int e = centry[u], l = e % Lb, k = e / Lb;
                const double w = wgt(l, k) * La;
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[q] += dfl[9 * l + q] * w;
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) a.band_df[9 * (size_t)b + q] = acc[q];
        }
    }
    __syncthreads();
    for (int l = threadIdx.x; l < Lb; l += blockDim.x) {
        if (a.Lux) a.Lux[l] = sh.Lux[l];
        if (a.Luy) a.Luy[l] = sh.Luy[l];
        if (a.Lfx) a.Lfx[l] = sh.Lfx[l];
        if (a.Lfy) a.Lfy[l] = sh.Lfy[l];
    }
    if (threadIdx.x == 0) {
        a.stats[4] = ST_OK;
        if (a.step_counter) *a.step_counter = s_step + 1;
    }
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_ibm_smem_bytes(int lb_total) { return (int)ibm_smem_bytes(lb_total); }

extern "C" int iblbm_ibm_scratch_doubles(int lb_total, int band_capacity, int n_particles)
{
    (void)n_particles;
    return 15 * band_capacity + 9 * lb_total;
}

extern "C" int iblbm_ibm_scratch_ints(int lb_total, int band_capacity, int box_capacity)
{
    (void)box_capacity;
    return 2 * band_capacity + 1 + MAX_S * lb_total;
}

extern "C" int iblbm_ibm_step_f64(const iblbm_ibm_args* a, void* stream)
{
    if (!a || !a->moff || a->n_particles < 1 || a->lb_total < 1 || !a->fpost_prev || !a->box || !a->map ||
        !a->band_nodes || !a->band_count || !a->scratch || !a->iscratch || !a->stats || !a->dstats || !a->larea)
        return IBLBM_E_ARG;
    if (a->delta_type != 0 && a->delta_type != 1) return IBLBM_E_ARG;
    if (a->method != IBM_DF && a->method != IBM_MDF && a->method != IBM_DFC) return IBLBM_E_ARG;
    if ((a->method == IBM_DF || a->method == IBM_MDF) && !a->band_fib) return IBLBM_E_ARG;
    if (a->method == IBM_DFC && (!a->band_df || !a->lambda || a->n_particles != 1)) return IBLBM_E_ARG;
    if (!a->xt_table && (!a->Lx || !a->Ly || !a->dvel)) return IBLBM_E_ARG;
    if (a->xt_table && (!a->Lx_c || !a->Ly_c || !a->step_counter || a->xt_len < 1)) return IBLBM_E_ARG;
    if ((a->c.bc == BC_OPEN || a->c.bc == BC_VELOCITY_INLET) && !a->uring_prev) return IBLBM_E_ARG;
    if (a->band_capacity < 1 || a->g.nx < 4 || a->g.ny < 4) return IBLBM_E_ARG;
    const size_t smem = ibm_smem_bytes(a->lb_total);
    if (smem > 220 * 1024) return IBLBM_E_CAPACITY;
    static int configured = 0;
    if (!configured) {
        if (cudaFuncSetAttribute(ibm_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024) !=
            cudaSuccess)
            return IBLBM_E_LAUNCH;
        configured = 1;
    }
    CollParams cp;
    BcParams bc;
    make_params(a->c, cp, bc);
    ibm_step_kernel<<<1, IBM_THREADS, smem, (cudaStream_t)stream>>>(*a, bc);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}
