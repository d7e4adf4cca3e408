// particles_f64.cu — rigid-particle update of sedimentation runs on the device.
//
// The Velocity-Verlet Newton-Euler step of runtime/scenarios/sedimentation_multi.py
// (:36-80 half step, :83-111 full step) for up to 8 discs, in FP64 without
// multiply-add contraction, with the same scalar expressions as the host step:
//   half  F = F_h + G;  v_half = v + (0.5 dt) F / m [+ 0.5 c (v - v_prev)];
//         x_next = x + (dt v_half) dx;  [omega_half = omega + (0.5 dt) T / I;
//         angle += dt omega_half];  markers X = R(angle) (X_c - X_0) + x_next;
//         desired velocity v_half [+ omega x (X - x_next) / dx, semi-implicit]
//   full  F_h = -sum over the band of the particle's spread force;
//         [T = -sum of (i - x/dx) fy - (j - y/dy) fx;  omega = omega_half +
//         (0.5 dt) T / I];
//         v_new = v_half + (0.5 dt) (F_h + G) / m [+ 0.5 c (v - v_prev)]
//         [+ (1 / rho_ratio) (v - v_prev)];  v_prev = v;  v = v_new;  x = x_next
// (c = pi r^2 / m for the explicit-history inertia model, physics/inertia/
// explicit_history.py:53-66; the rho-ratio term for feng_b2, feng_b2.py:33-48;
// the angular kicks of physics/rigid_body.py:65-82, the marker rotation of
// physics/markers.py:23-38 and the rigid-body velocity of :41-60).
// One launch after the band kernel does the full step of this timestep and the
// half step of the next, so the whole step stays on the device and can be
// captured in a CUDA graph.  The explicit Euler step (sedimentation_multi.py:
// 126-190) is one launch after the band kernel too (after the whole lattice
// pass when rotating):
//   [L = the fluid's angular momentum inside the disc from this step's rho, U;
//   omega_new = omega + (L - L_prev + dt T) / I;  angle += dt omega_new, or
//   0.5 dt (omega + omega_new) (trapezoidal)];
//   v_new = v + dt F / m [+ c (v - v_prev)];  x_new = x + (dt v_new) dx, or
//   x + (0.5 dt (v + v_new)) dx (trapezoidal);  [v_new += (1 / rho_ratio)
//   (v - v_prev)];  then the next step's markers at x_new (turned by the
//   angle), desired velocity v_new [+ omega_new x r].
//
// The force is -sum of the particle's spread force over the lattice.  The
// reference sums its dense n_nodes x 2 field with numpy (np.sum: pairwise
// summation, iblbm/ibm/multi_particle.py:199-202); given that summation tree
// (pw_* fields, built on the host from n_nodes) the kernel evaluates it over
// the band's nonzero entries: every block of the tree sums its entries in
// numpy's order (8 strided accumulators, their fixed combination, the tail),
// a block without band entries sums to +0.0, and the inner nodes add their
// children level by level.  Adding the zeros numpy adds would change no
// partial sum, so the force equals numpy's bit for bit and the trajectories
// equal the host step's.  The torque is the same pairwise sum of its dense
// moment-arm field (:203-208; its zero terms may be -0.0, which changes no
// partial sum that is not itself zero).  Without a tree the sums run in
// another fixed order (deterministic, round-off apart from numpy's).  The
// rotated markers take the device's cos and sin of the angle, which may differ
// from the host's in the last bit, so rotating runs are not bit for bit.  DF and
// DFC particles take their forces and torques from their markers' forces
// instead, each a pairwise sum over the particle's markers (lagrangian_sums).
#include <cstdint>
#include "common.cuh"
#include "../../include/iblbm_b200.h"

namespace iblbm {

constexpr int PART_THREADS = 256;
constexpr int PART_MAXP = 8;
constexpr int PART_MAXB = 2048;  // band capacity limit of the band kernel

// channel pc of the sums at band entry b (lattice index e): the force
// components of the particles (pc < 2P), then their torque terms
template <typename F>
__device__ __forceinline__ double channel_value(const iblbm_particles_args& a, const F* fib, size_t pstride,
                                                const double* s_ctr, int pc, int b, int e)
{
    const int P2 = 2 * a.n_particles;
    if (pc < P2) return (double)fib[(pc >> 1) * pstride + 2 * (size_t)b + (pc & 1)];
    const int p = pc - P2;
    const double fx = (double)fib[p * pstride + 2 * (size_t)b];
    const double fy = (double)fib[p * pstride + 2 * (size_t)b + 1];
    const double i = (double)(e % a.nx), j = (double)(e / a.nx);
    return (i - s_ctr[2 * p]) * fy - (j - s_ctr[2 * p + 1]) * fx;
}

template <typename F>
__device__ void particle_forces(const iblbm_particles_args& a, const F* fib, const double* s_ctr, int PC,
                                double* s_force)
{
    __shared__ double red[PART_THREADS];
    const int nb = *a.band_count;
    const size_t pstride = 2 * (size_t)a.band_capacity;
    for (int pc = 0; pc < PC; ++pc) {
        double sum = 0.0;
        for (int b = threadIdx.x; b < nb; b += PART_THREADS)
            sum += channel_value(a, fib, pstride, s_ctr, pc, b, pc < 2 * a.n_particles ? 0 : a.band_nodes[b]);
        red[threadIdx.x] = sum;
        __syncthreads();
        for (int w = PART_THREADS / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) s_force[pc] = -red[0];
        __syncthreads();
    }
}

// numpy's pairwise sum of the dense field, over the band entries only (see the
// file comment).  The band's lattice indices go to shared memory; only the
// leaves between the band's first and last index (the window, found through
// pw_lut) are summed, and an inner node outside the window is +0.0, which its
// parent adds like numpy adds the sum of a block of zeros.
__device__ __forceinline__ int pw_leaf_of(const iblbm_particles_args& a, int e)
{
    int l = a.pw_lut[e >> 6];
    if (l + 1 < a.pw_leaves && a.pw_leaf[2 * (l + 1)] <= e) ++l;
    return l;
}

constexpr int PW_MAXLEVELS = 64;
constexpr int PW_SV = 6144;  // window partial sums held in shared memory (doubles)
constexpr int PW_SN = 2048;  // window inner nodes whose children are held in shared memory
// two particles' band forces, the window's partial sums and its inner nodes' children
constexpr size_t PART_DYN_SMEM = (4 * PART_MAXB + PW_SV) * sizeof(double) + 2 * PW_SN * sizeof(int);

// first k in [A, B) with pred(k) (pred false then true along k), B if none:
// the 32 lanes of a warp probe 32 evenly spaced points per round
template <typename Pred>
__device__ int warp_first_true(int A, int B, Pred pred)
{
    const int lane = threadIdx.x & 31;
    int lo = A, hi = B;  // the answer lies in [lo, hi]
    while (lo < hi) {
        const int step = (hi - lo + 31) / 32;
        const int k = lo + lane * step;
        const unsigned m = __ballot_sync(0xffffffffu, k < hi && pred(k));
        if (m) {
            const int j = __ffs(m) - 1;
            hi = lo + j * step;
            if (j) lo += (j - 1) * step + 1;
        } else {  // every probe below hi was false
            lo += ((hi - 1 - lo) / step) * step + 1;
        }
    }
    return lo;
}

template <typename F>
__device__ void particle_forces_exact(const iblbm_particles_args& a, const F* fib, const double* s_ctr, int PC,
                                      double* s_force, double* s_f)
{
    __shared__ int s_nodes[PART_MAXB];
    const int nb = min(*a.band_count, PART_MAXB);
    const int P = a.n_particles, L = a.pw_leaves;
    const size_t pstride = 2 * (size_t)a.band_capacity;
    double* v = a.pw_scratch;  // node id x PC
    for (int b = threadIdx.x; b < nb; b += PART_THREADS) s_nodes[b] = a.band_nodes[b];
    __syncthreads();
    if (nb == 0) {
        if (threadIdx.x < PC) s_force[threadIdx.x] = -(0.0 + 0.0);
        __syncthreads();
        return;
    }
    const int l0 = pw_leaf_of(a, s_nodes[0]), l1 = pw_leaf_of(a, s_nodes[nb - 1]);
    // a level's nodes are disjoint and left to right, so those meeting the window
    // are one run [s_klo, s_kend); one warp per level finds it
    __shared__ int s_klo[PW_MAXLEVELS], s_kend[PW_MAXLEVELS], s_base[PW_MAXLEVELS + 1];
    for (int d = (int)threadIdx.x >> 5; d < a.pw_levels; d += PART_THREADS / 32) {
        const int A = a.pw_level[d], B = a.pw_level[d + 1];
        const int klo = warp_first_true(A, B, [&](int k) { return a.pw_span[2 * k + 1] >= l0; });
        const int kend = warp_first_true(klo, B, [&](int k) { return a.pw_span[2 * k] > l1; });
        if ((threadIdx.x & 31) == 0) {
            s_klo[d] = klo;
            s_kend[d] = kend;
        }
    }
    __syncthreads();
    // window-local ids: the window's leaves first, then its inner nodes level by level
    const int WL = l1 - l0 + 1;
    if (threadIdx.x == 0) {
        int t = WL;
        for (int d = 0; d < a.pw_levels; ++d) {
            s_base[d] = t;
            t += s_kend[d] - s_klo[d];
        }
        s_base[a.pw_levels] = t;
    }
    __syncthreads();
    const int WN = s_base[a.pw_levels];  // window nodes, leaves included
    // the partial sums of the window live in shared memory when they fit (sv:
    // PW_SV doubles; lc: the window-local children of up to PW_SN inner nodes),
    // else in the global scratch v
    const bool fast = (size_t)WN * PC <= PW_SV && WN - WL <= PW_SN;
    double* sv = s_f + 4 * PART_MAXB;
    int* lc = reinterpret_cast<int*>(sv + PW_SV);
    auto vref = [&](int li, int pc) -> double& { return fast ? sv[(li - l0) * PC + pc] : v[(size_t)li * PC + pc]; };
    // two particles at a time: their band forces staged in shared memory (s_f: fx,
    // fy of the first, then of the second, PART_MAXB each), so the leaves' ordered
    // sums read no global memory and each leaf's entries are walked once per pair
    const bool rot = a.rotation != 0;
    for (int p0 = 0; p0 < P; p0 += 2) {
        const int np = min(2, P - p0);
        for (int b = threadIdx.x; b < nb; b += PART_THREADS)
            for (int q = 0; q < np; ++q) {
                s_f[(2 * q) * PART_MAXB + b] = (double)fib[(p0 + q) * pstride + 2 * (size_t)b];
                s_f[(2 * q + 1) * PART_MAXB + b] = (double)fib[(p0 + q) * pstride + 2 * (size_t)b + 1];
            }
        __syncthreads();
        double cx[2], cy[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            cx[q] = q < np ? s_ctr[2 * (p0 + q)] : 0.0;
            cy[q] = q < np ? s_ctr[2 * (p0 + q) + 1] : 0.0;
        }
        for (int li = l0 + (int)threadIdx.x; li <= l1; li += PART_THREADS) {
            const int off = a.pw_leaf[2 * li], m = a.pw_leaf[2 * li + 1];
            int b = 0, hi = nb;  // first band entry at or after off
            while (b < hi) {
                const int mid = (b + hi) >> 1;
                if (s_nodes[mid] < off) b = mid + 1;
                else hi = mid;
            }
            // channel 3 q + c of particle p0 + q: c = 0 fx, 1 fy, 2 the torque term
            // (i - cx) fy - (j - cy) fx; entry e's terms added to accumulator k
            double res[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) res[c] = 0.0;
            auto add = [&](int e, double (&acc)[6]) {
                double i = 0.0, j = 0.0;
                if (rot) {
                    const int n = s_nodes[e];
                    i = (double)(n % a.nx);
                    j = (double)(n / a.nx);
                }
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (q < np) {
                        const double fx = s_f[(2 * q) * PART_MAXB + e], fy = s_f[(2 * q + 1) * PART_MAXB + e];
                        acc[3 * q] += fx;
                        acc[3 * q + 1] += fy;
                        if (rot) acc[3 * q + 2] += (i - cx[q]) * fy - (j - cy[q]) * fx;
                    }
                }
            };
            if (m >= 8) {
                // numpy's 8 strided accumulators, in registers: the entries of each
                // 8-position block go to the lanes of their positions, in order
                const int cut = off + (m - m % 8);
                double r[8][6];
#pragma unroll
                for (int k = 0; k < 8; ++k)
#pragma unroll
                    for (int c = 0; c < 6; ++c) r[k][c] = 0.0;
                while (b < nb && s_nodes[b] < cut) {
                    const int q0 = off + ((s_nodes[b] - off) & ~7);
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        if (b < nb && s_nodes[b] == q0 + k) {
                            add(b, r[k]);
                            ++b;
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    res[c] = ((r[0][c] + r[1][c]) + (r[2][c] + r[3][c])) + ((r[4][c] + r[5][c]) + (r[6][c] + r[7][c]));
            }
            for (; b < nb && s_nodes[b] < off + m; ++b) add(b, res);  // the tail (or a leaf of under 8)
            for (int q = 0; q < np; ++q) {
                vref(li, 2 * (p0 + q)) = res[3 * q];
                vref(li, 2 * (p0 + q) + 1) = res[3 * q + 1];
                if (rot) vref(li, 2 * P + p0 + q) = res[3 * q + 2];
            }
        }
        __syncthreads();
    }
    // a child is in the window when its leaves meet [l0, l1]; outside it sums to +0.0
    auto in_window = [&](int id) {
        if (id < L) return id >= l0 && id <= l1;
        const int k = id - L;
        return a.pw_span[2 * k + 1] >= l0 && a.pw_span[2 * k] <= l1;
    };
    const int root = a.pw_internal > 0 ? L + a.pw_internal - 1 : 0;
    if (fast) {
        // window-local ids of the children of every window inner node (-1: outside
        // the window, adds +0.0), read once, then the levels in shared memory
        auto local = [&](int id) {
            if (id < L) return id >= l0 && id <= l1 ? id - l0 : -1;
            const int k = id - L;
            for (int d = 0; d < a.pw_levels; ++d)
                if (k >= s_klo[d] && k < s_kend[d]) return s_base[d] + k - s_klo[d];
            return -1;
        };
        for (int u = WL + (int)threadIdx.x; u < WN; u += PART_THREADS) {
            int d = 0;
            while (u >= s_base[d + 1]) ++d;
            const int k = s_klo[d] + u - s_base[d];
            lc[2 * (u - WL)] = local(a.pw_node[2 * k]);
            lc[2 * (u - WL) + 1] = local(a.pw_node[2 * k + 1]);
        }
        __syncthreads();
        for (int d = 0; d < a.pw_levels; ++d) {  // one thread per node and channel
            const int n0 = s_base[d], cnt = (s_base[d + 1] - n0) * PC;
            for (int x = threadIdx.x; x < cnt; x += PART_THREADS) {
                const int u = n0 + x / PC, pc = x % PC;
                const int c0 = lc[2 * (u - WL)], c1 = lc[2 * (u - WL) + 1];
                const double x0 = c0 >= 0 ? sv[c0 * PC + pc] : 0.0;
                const double x1 = c1 >= 0 ? sv[c1 * PC + pc] : 0.0;
                sv[u * PC + pc] = x0 + x1;
            }
            __syncthreads();
        }
        // the root meets the window (it holds every leaf)
        const int r = local(root);
        if (threadIdx.x < PC) s_force[threadIdx.x] = -(0.0 + sv[r * PC + threadIdx.x]);
    } else {
        for (int d = 0; d < a.pw_levels; ++d) {
            for (int k = s_klo[d] + threadIdx.x; k < s_kend[d]; k += PART_THREADS) {
                const int c0 = a.pw_node[2 * k], c1 = a.pw_node[2 * k + 1];
                const bool w0 = in_window(c0), w1 = in_window(c1);
                for (int pc = 0; pc < PC; ++pc) {
                    const double x0 = w0 ? v[(size_t)c0 * PC + pc] : 0.0;
                    const double x1 = w1 ? v[(size_t)c1 * PC + pc] : 0.0;
                    v[(size_t)(L + k) * PC + pc] = x0 + x1;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x < PC) s_force[threadIdx.x] = -(0.0 + v[(size_t)root * PC + threadIdx.x]);
    }
    __syncthreads();
}

// numpy's pairwise summation of n values (the tree of the file comment):
// leaves of at most 128 values, each summed in 8 strided accumulators and a
// tail, a longer range split at half its length rounded down to a multiple of 8
__device__ double pw_block(const double* v, int n)
{
    if (n < 8) {
        double res = 0.0;
        for (int i = 0; i < n; ++i) res += v[i];
        return res;
    }
    double r[8];
    for (int k = 0; k < 8; ++k) r[k] = v[k];
    int i = 8;
    for (; i < n - n % 8; i += 8)
        for (int k = 0; k < 8; ++k) r[k] += v[i + k];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += v[i];
    return res;
}

__device__ void pw_collect(int off, int n, int* loff, int* llen, int& cnt)
{
    if (n <= 128) {
        loff[cnt] = off;
        llen[cnt] = n;
        ++cnt;
        return;
    }
    int n2 = n / 2;
    n2 -= n2 % 8;
    pw_collect(off, n2, loff, llen, cnt);
    pw_collect(off + n2, n - n2, loff, llen, cnt);
}

__device__ double pw_fold(int n, const double* lsum, int& li)
{
    if (n <= 128) return lsum[li++];
    int n2 = n / 2;
    n2 -= n2 % 8;
    const double x = pw_fold(n2, lsum, li);
    const double y = pw_fold(n - n2, lsum, li);
    return x + y;
}

constexpr int PW_MAXLEAVES = 512;  // every leaf but a lone one holds at least 64 values
constexpr int LINT_MAX = 64 * (PW_MAXLEAVES - 1);

// numpy's pairwise sum of vals[0 .. n), n <= LINT_MAX (global memory the block
// wrote before a __syncthreads); block-wide, the sum is returned to thread 0
__device__ double block_pairwise_sum(const double* vals, int n)
{
    __shared__ int s_nleaves;
    __shared__ int s_loff[PW_MAXLEAVES], s_llen[PW_MAXLEAVES];
    __shared__ double s_lsum[PW_MAXLEAVES];
    if (threadIdx.x == 0) {
        int cnt = 0;
        if (n > 0) pw_collect(0, n, s_loff, s_llen, cnt);
        s_nleaves = cnt;
    }
    __syncthreads();
    for (int l = threadIdx.x; l < s_nleaves; l += PART_THREADS) s_lsum[l] = pw_block(vals + s_loff[l], s_llen[l]);
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0 && n > 0) {
        int li = 0;
        total = pw_fold(n, s_lsum, li);
    }
    __syncthreads();
    return total;
}

// The fluid's angular momentum inside a disc (centre px, py, radius r) from
// this step's rho and U: diagnostics/internal_flow.py:220-262 as the host
// restates it — the box of half-width int(r/dx) + 2 around the rounded centre
// (round half to even), clipped to the lattice, the nodes with
// RX^2 + RY^2 <= (r/dx)^2 in row order, each value (RX rho) uy - (RY rho) ux,
// summed pairwise.  Block-wide; the sum is returned to thread 0.
template <typename T>
__device__ double disc_angular_momentum(const iblbm_particles_args& a, const T* rho, const T* U, double px,
                                        double py, double r)
{
    __shared__ int s_base;
    __shared__ int s_wcount[PART_THREADS / 32];
    const double dx = a.dx;
    const double ci = px / dx, cj = py / dx, rl = r / dx;
    const int ii = (int)rint(ci), jj = (int)rint(cj), rr = (int)rl + 2;
    const int i0 = max(0, ii - rr), i1 = min(a.nx, ii + rr + 1);
    const int j0 = max(0, jj - rr), j1 = min(a.ny, jj + rr + 1);
    const int W = max(0, i1 - i0), H = max(0, j1 - j0), nbox = W * H;
    const double r2 = rl * rl;
    const int cap = min(a.lint_capacity, LINT_MAX);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < nbox; c0 += PART_THREADS) {
        const int k = c0 + (int)threadIdx.x;
        bool in = false;
        double val = 0.0;
        if (k < nbox) {
            const int i = i0 + k % W, j = j0 + k / W;
            const double RX = (double)i - ci, RY = (double)j - cj;
            in = RX * RX + RY * RY <= r2;
            if (in) {
                const size_t e = (size_t)j * a.nx + i;
                const double ro = (double)rho[e], ux = (double)U[2 * e], uy = (double)U[2 * e + 1];
                val = (RX * ro) * uy - (RY * ro) * ux;
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (lane == 0) s_wcount[w] = __popc(bal);
        __syncthreads();
        int off = s_base + __popc(bal & ((1u << lane) - 1u));
        for (int q = 0; q < w; ++q) off += s_wcount[q];
        if (in && off < cap) a.lint_scratch[off] = val;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = s_base;
            for (int q = 0; q < PART_THREADS / 32; ++q) t += s_wcount[q];
            s_base = t;
        }
        __syncthreads();
    }
    return block_pairwise_sum(a.lint_scratch, min(s_base, cap));
}

// Each particle's force and torque from its markers' forces, summed like the
// reference: DF (iblbm/ibm/forcing.py:262-275) F = -sum(Lf ds), T =
// -sum((rx Lfy - ry Lfx) ds); DFC (iblbm/ibm/strategies/dfc.py:114-128) F =
// sum(f), T = sum(rx fy - ry fx); rx = (X - x)/dx, ry = (Y - y)/dy over the
// markers of this step, each sum numpy's pairwise sum of the particle's values.
__device__ void lagrangian_sums(const iblbm_particles_args& a, double* s_force)
{
    const int P = a.n_particles;
    const bool rot = a.rotation != 0, df = a.lagrangian == IBLBM_LAGRANGIAN_DF;
    const int cap = min(a.lint_capacity, LINT_MAX);
    double* buf = a.lint_scratch;
    for (int p = 0; p < P; ++p) {
        const int m0 = a.moff[p], n = min(a.moff[p + 1] - m0, cap);
        const double* st = a.state + IBLBM_PARTICLE_STATE * p;
        const double px = st[10], py = st[11];
        const double ds = a.consts[IBLBM_PARTICLE_CONSTS * p + 9];
        for (int c = 0; c < (rot ? 3 : 2); ++c) {
            for (int l = threadIdx.x; l < n; l += PART_THREADS) {
                const int m = m0 + l;
                const double fx = df ? a.Lfx[m] : a.dfc_force[2 * m];
                const double fy = df ? a.Lfy[m] : a.dfc_force[2 * m + 1];
                double v;
                if (c < 2) {
                    v = c == 0 ? fx : fy;
                } else {
                    const double rx = (a.Lx[m] - px) / a.dx, ry = (a.Ly[m] - py) / a.dy;
                    v = rx * fy - ry * fx;
                }
                buf[l] = df ? v * ds : v;
            }
            __syncthreads();
            const double t = 0.0 + block_pairwise_sum(buf, n);
            if (threadIdx.x == 0) s_force[c < 2 ? 2 * p + c : 2 * P + p] = df ? -t : t;
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(PART_THREADS) particles_kernel(const iblbm_particles_args a)
{
    __shared__ double s_force[3 * PART_MAXP];  // forces (2 per particle), then torques
    __shared__ double s_ctr[2 * PART_MAXP];    // the centres in lattice units, for the torques
    __shared__ double s_next[2 * PART_MAXP], s_vh[2 * PART_MAXP];
    __shared__ double s_rot[3 * PART_MAXP];    // cos, sin of the angle; omega of the rigid-body velocity
    __shared__ double s_lint[PART_MAXP];       // the fluid's angular momentum inside each disc
    const int P = a.n_particles;
    const double dt = a.dt, dx = a.dx;
    if (a.phase & (IBLBM_PARTICLES_FULL | IBLBM_PARTICLES_EULER)) {
        const int PC = 2 * P + (a.rotation ? P : 0);
        if (threadIdx.x < 2 * P) {
            const int p = threadIdx.x >> 1, d = threadIdx.x & 1;
            s_ctr[threadIdx.x] = a.state[IBLBM_PARTICLE_STATE * p + 10 + d] / (d ? a.dy : dx);
        }
        __syncthreads();
        if (a.lagrangian) {
            lagrangian_sums(a, s_force);
        } else if (a.pw_leaf) {
            extern __shared__ double s_dyn[];  // PART_DYN_SMEM bytes with a summation tree
            if (a.fib_f32)
                particle_forces_exact(a, static_cast<const float*>(a.band_fib_part), s_ctr, PC, s_force, s_dyn);
            else
                particle_forces_exact(a, static_cast<const double*>(a.band_fib_part), s_ctr, PC, s_force, s_dyn);
        } else if (a.fib_f32) {
            particle_forces(a, static_cast<const float*>(a.band_fib_part), s_ctr, PC, s_force);
        } else {
            particle_forces(a, static_cast<const double*>(a.band_fib_part), s_ctr, PC, s_force);
        }
    }
    if (a.phase & IBLBM_PARTICLES_FULL) {
        if (threadIdx.x < P) {
            const int p = threadIdx.x;
            double* s = a.state + IBLBM_PARTICLE_STATE * p;
            const double* c = a.consts + IBLBM_PARTICLE_CONSTS * p;
            const double m = c[0], inv_rho = c[1], hc = c[2];
            // this step's half-step values become current (the half step wrote them ahead)
            s[6] = s[16];
            s[7] = s[17];
            if (a.rotation) {  // physics/rigid_body.py:77-82
                s[13] = s[18];
                s[14] = s[19];
                s[20] = s[12];  // the omega this step's half step turned its markers with
                const double T = s_force[2 * P + p];
                s[12] = s[13] + ((0.5 * dt) * T) / c[7];
                s[15] = T;
            }
            for (int d = 0; d < 2; ++d) {
                if (a.prescribed) {  // sedimentation_single.py:174-180: the velocity stays
                    s[2 + d] = a.prescribed_velocity[d];
                    s[8 + d] = s_force[2 * p + d];
                    s[d] = s[10 + d];
                    if (a.forces_out) a.forces_out[2 * p + d] = s_force[2 * p + d];
                    continue;
                }
                const double F = s_force[2 * p + d] + c[3 + d];
                double vn = s[6 + d] + ((0.5 * dt) * F) / m;
                if (a.model == IBLBM_INERTIA_EXPLICIT_HISTORY) vn = vn + 0.5 * (hc * (s[2 + d] - s[4 + d]));
                if (a.model == IBLBM_INERTIA_FENG_B2) vn = vn + inv_rho * (s[2 + d] - s[4 + d]);
                s[4 + d] = s[2 + d];      // v_prev = v
                s[2 + d] = vn;            // v
                s[8 + d] = s_force[2 * p + d];
                s[d] = s[10 + d];         // x = x_next
                if (a.forces_out) a.forces_out[2 * p + d] = s_force[2 * p + d];
            }
        }
        __syncthreads();
    }
    if (a.phase & IBLBM_PARTICLES_EULER) {
        if (a.rotation) {
            for (int p = 0; p < P; ++p) {
                const double* s = a.state + IBLBM_PARTICLE_STATE * p;
                const double r = a.consts[IBLBM_PARTICLE_CONSTS * p + 8];
                const double l = a.moments_f32
                    ? disc_angular_momentum(a, static_cast<const float*>(a.rho), static_cast<const float*>(a.U),
                                            s[0], s[1], r)
                    : disc_angular_momentum(a, static_cast<const double*>(a.rho), static_cast<const double*>(a.U),
                                            s[0], s[1], r);
                if (threadIdx.x == 0) s_lint[p] = 0.0 + l;
            }
            __syncthreads();
        }
        if (threadIdx.x < P) {
            const int p = threadIdx.x;
            double* s = a.state + IBLBM_PARTICLE_STATE * p;
            const double* c = a.consts + IBLBM_PARTICLE_CONSTS * p;
            const double m = c[0], inv_rho = c[1], hc = c[2];
            for (int d = 0; d < 2; ++d) {
                const double F = s_force[2 * p + d] + c[3 + d];
                double vn = s[2 + d] + (dt * F) / m;
                if (a.model == IBLBM_INERTIA_EXPLICIT_HISTORY) vn = vn + hc * (s[2 + d] - s[4 + d]);
                const double xn = a.euler_trapezoidal ? s[d] + ((0.5 * dt) * (s[2 + d] + vn)) * dx
                                                      : s[d] + (dt * vn) * dx;
                if (a.model == IBLBM_INERTIA_FENG_B2) vn = vn + inv_rho * (s[2 + d] - s[4 + d]);
                s[4 + d] = s[2 + d];      // v_prev = v
                s[2 + d] = vn;            // v
                s[6 + d] = vn;
                s[16 + d] = vn;
                s[8 + d] = s_force[2 * p + d];
                s[d] = xn;
                s[10 + d] = xn;
                s_vh[2 * p + d] = vn;
                s_next[2 * p + d] = xn;
                if (a.forces_out) a.forces_out[2 * p + d] = s_force[2 * p + d];
            }
            if (a.rotation) {  // physics/rigid_body.py:101-121
                const double T = s_force[2 * P + p];
                const double dl = s_lint[p] - s[21];
                s[21] = s_lint[p];
                const double om = s[12] + (dl + dt * T) / c[7];
                s[14] = a.euler_trapezoidal ? s[14] + (0.5 * dt) * (s[12] + om) : s[14] + dt * om;
                s[15] = T;
                s[12] = om;
                s[19] = s[14];
            }
            // R(0) = [[1, -0], [0, 1]] exactly, as the host's cos 0 and sin 0
            s_rot[3 * p] = a.rotation ? cos(s[14]) : 1.0;
            s_rot[3 * p + 1] = a.rotation ? sin(s[14]) : 0.0;
            s_rot[3 * p + 2] = a.rotation ? s[12] : 0.0;
        }
        __syncthreads();
    }
    if (a.phase & IBLBM_PARTICLES_HALF) {
        if (threadIdx.x < P) {
            const int p = threadIdx.x;
            double* s = a.state + IBLBM_PARTICLE_STATE * p;
            const double* c = a.consts + IBLBM_PARTICLE_CONSTS * p;
            const double m = c[0], hc = c[2];
            for (int d = 0; d < 2; ++d) {
                const double F = s[8 + d] + c[3 + d];
                double vh = s[2 + d] + ((0.5 * dt) * F) / m;
                if (a.model == IBLBM_INERTIA_EXPLICIT_HISTORY) vh = vh + 0.5 * (hc * (s[2 + d] - s[4 + d]));
                if (a.prescribed) vh = a.prescribed_velocity[d];  // sedimentation_single.py:91-97
                const double xn = s[d] + (dt * vh) * dx;
                s[16 + d] = vh;
                s[10 + d] = xn;
                s_vh[2 * p + d] = vh;
                s_next[2 * p + d] = xn;
            }
            if (a.rotation) {  // physics/rigid_body.py:65-74
                s[18] = s[12] + ((0.5 * dt) * s[15]) / c[7];
                s[19] = s[14] + dt * s[18];
            }
            // R(0) = [[1, -0], [0, 1]] exactly, as the host's cos 0 and sin 0
            s_rot[3 * p] = a.rotation ? cos(s[19]) : 1.0;
            s_rot[3 * p + 1] = a.rotation ? sin(s[19]) : 0.0;
            s_rot[3 * p + 2] = a.rotation && a.semi_implicit ? (a.half_kick_omega ? s[18] : s[12]) : 0.0;
        }
        __syncthreads();
    }
    if (a.phase & (IBLBM_PARTICLES_HALF | IBLBM_PARTICLES_EULER)) {
        const int Lb = a.moff[P];
        for (int l = threadIdx.x; l < Lb; l += PART_THREADS) {
            int p = 0;
            while (p + 1 < P && l >= a.moff[p + 1]) ++p;
            const double* c = a.consts + IBLBM_PARTICLE_CONSTS * p;
            const double rx = a.Lx_c[l] - c[5], ry = a.Ly_c[l] - c[6];
            const double cs = s_rot[3 * p], sn = s_rot[3 * p + 1], om = s_rot[3 * p + 2];
            const double X = (cs * rx - sn * ry) + s_next[2 * p];
            const double Y = (sn * rx + cs * ry) + s_next[2 * p + 1];
            double u = s_vh[2 * p], v = s_vh[2 * p + 1];
            if (om != 0.0) {  // U + omega x r, physics/markers.py:41-60
                u = u + ((-om) * (Y - s_next[2 * p + 1])) / dx;
                v = v + (om * (X - s_next[2 * p])) / dx;
            }
            a.Lx[l] = X;
            a.Ly[l] = Y;
            a.dvel[2 * l] = u;
            a.dvel[2 * l + 1] = v;
        }
    }
}

}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_particles_step_f64(const iblbm_particles_args* a, void* stream)
{
    if (!a || a->n_particles < 1 || a->n_particles > PART_MAXP || !a->moff || !a->state || !a->consts)
        return IBLBM_E_ARG;
    const int ph = a->phase;
    if ((ph & ~(IBLBM_PARTICLES_FULL | IBLBM_PARTICLES_HALF | IBLBM_PARTICLES_EULER)) || !ph) return IBLBM_E_ARG;
    if ((ph & IBLBM_PARTICLES_EULER) && ph != IBLBM_PARTICLES_EULER) return IBLBM_E_ARG;
    if ((ph & IBLBM_PARTICLES_EULER) && a->rotation &&
        (!a->rho || !a->U || a->ny < 1 || !a->lint_scratch || a->lint_capacity < 1 || a->lint_capacity > LINT_MAX))
        return IBLBM_E_ARG;
    if ((ph & (IBLBM_PARTICLES_FULL | IBLBM_PARTICLES_EULER)) &&
        (!a->band_fib_part || !a->band_count || a->band_capacity < 1))
        return IBLBM_E_ARG;
    if ((ph & (IBLBM_PARTICLES_HALF | IBLBM_PARTICLES_EULER)) &&
        (!a->Lx_c || !a->Ly_c || !a->Lx || !a->Ly || !a->dvel))
        return IBLBM_E_ARG;
    if (a->rotation && (!a->band_nodes || a->nx < 1 || !(a->dy > 0.0))) return IBLBM_E_ARG;
    if (a->lagrangian < 0 || a->lagrangian > IBLBM_LAGRANGIAN_DFC) return IBLBM_E_ARG;
    if (a->prescribed && (a->rotation || (ph & IBLBM_PARTICLES_EULER))) return IBLBM_E_ARG;
    if (a->lagrangian && (ph & (IBLBM_PARTICLES_FULL | IBLBM_PARTICLES_EULER)) &&
        (!a->lint_scratch || a->lint_capacity < 1 || a->lint_capacity > LINT_MAX || !a->Lx || !a->Ly ||
         (a->lagrangian == IBLBM_LAGRANGIAN_DF ? (!a->Lfx || !a->Lfy) : !a->dfc_force)))
        return IBLBM_E_ARG;
    if (a->model < IBLBM_INERTIA_NONE || a->model > IBLBM_INERTIA_FENG_B2) return IBLBM_E_ARG;
    if (a->pw_leaf && (!a->pw_node && a->pw_internal > 0)) return IBLBM_E_ARG;
    if (a->pw_leaf && (!a->band_nodes || !a->pw_scratch || !a->pw_level || !a->pw_lut || !a->pw_span ||
                       a->pw_leaves < 1 || a->pw_internal < 0 || a->pw_levels < 0 || a->n_nodes < 1))
        return IBLBM_E_ARG;
    if (a->pw_leaf && (a->band_capacity > PART_MAXB || a->pw_levels > PW_MAXLEVELS)) return IBLBM_E_CAPACITY;
    const size_t dyn = a->pw_leaf ? PART_DYN_SMEM : 0;
    // the staging buffer takes static + dynamic shared memory past 48 KB
    if (smem_limit_once<particles_kernel>((int)PART_DYN_SMEM) != cudaSuccess) return IBLBM_E_LAUNCH;
    particles_kernel<<<1, PART_THREADS, dyn, (cudaStream_t)stream>>>(*a);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}
