// band_cluster.cuh — the MDF band step of one fixed body spread over a
// thread-block cluster (FP64 form).
//
// One CTA holds the whole band in the single-CTA step; its MDF iterations wait
// on that one SM's shared-memory pipe (gathers of band velocities and marker
// forces) and on long per-thread chains.  Here the body's markers are split
// into C contiguous ranges,
// one per CTA of a cluster of C CTAs on C SMs.  CTA c owns
//   * its markers [m0, m1): their stencil slots (CTA-local node, weight);
//   * its nodes: every band node under one of its markers' stencils, with that
//     node's contribution list (marker, weight) in shared memory.
// Both sit in shared memory, one column per thread, and are walked by
// straight-line code (the whole stencil; a list's first CL_JU entries,
// predicated on its length) so that their loads issue ahead of the serial sums:
// measured standalone, a stencil walked one row per loop trip takes twice as
// long as the unrolled one.
// A node under the stencils of markers of two CTAs is held by both; both run
// the same operations on the same inputs, so both copies keep the same bits.
// An iteration is
//   interpolate + slip + force (marker threads, from the CTA's own nodes)
//   -> each marker's force stored into every CTA's shared memory, and each
//      marker warp's maximum squared slip into a slot of every CTA
//   -> cluster barrier (release / acquire)
//   -> spread + relax + velocity update (node threads, forces of any marker
//      read from the CTA's own copy), while one warp reduces the residual =
//      sqrt of the maximum over the slots (the same bits in every CTA, so
//      every CTA takes the same branch)
//   -> CTA barrier -> divergence check (a diverged iteration's spread is
//      undone: its force increments are dropped) -> convergence check.
// Every sum runs over the same terms in the same order as the single-CTA step
// (slot order for interpolation, list order for spreading), so every result is
// bit-identical to it.  The force copies and residual slots are double-buffered
// by iteration parity: a CTA that runs ahead writes the other buffer, and cannot
// come back to this one before every CTA has passed the next cluster barrier.
//
// The per-CTA plan (marker ranges, node sets, lists, slot order) is built from
// the body's cached lists by ibm_cluster_plan_kernel right after each band
// rebuild.  When the plan does not hold (a list longer than the stencil, from
// stencil slots clamped onto an edge node; more nodes under a rank's markers
// than the CTA has threads left; or no band), the cluster's first CTA
// runs the single-CTA step instead and the others return, so the launch always
// computes the step.
//
// Every CTA of the cluster reaches every cluster barrier the same number of
// times: each branch around one depends only on values that are identical in
// all CTAs (the plan header, the iteration count, and the residual, which every
// CTA reduces from the same slots).  No TMA or multicast; the only remote
// accesses are plain shared::cluster stores.
#pragma once
#include <algorithm>
#include "band_kernel.cuh"

namespace iblbm {

constexpr int CL_MAX = 8;     // CTAs per cluster (the portable cluster size)
constexpr int CL_HDR = 16;    // plan header ints: [C, S, Lb, nb, NMP, NLP, 0, 0, rank status x CL_MAX]
constexpr int CL_JU = 8;      // list entries of a node spread by straight-line code

// Plan sizes of one rank: markers per CTA (capacity NMP), nodes per CTA
// (capacity NLP: the most distinct nodes the markers can cover, at most the
// CTA's threads after its marker warps; a band whose ranks find more nodes
// than that takes the single-CTA fallback).
struct ClusterDims {
    int C, S, SW, nm, MW, NMP, NLP, rank_ints;
};

__host__ __device__ inline int cl_up2(int x) { return (x + 1) & ~1; }

__host__ __device__ inline ClusterDims cluster_dims(int Lb, int S, int C)
{
    ClusterDims d;
    d.C = C;
    d.S = S;
    d.nm = (Lb + C - 1) / C;
    d.MW = (d.nm + 31) / 32;
    d.NMP = cl_up2(d.nm);
    // node capacity: the nodes the markers can cover, at most the CTA's threads
    // after the marker warps (the plan checks the count it finds against it)
    const int cover = d.nm * S, room = IBM_THREADS - 32 * d.MW;
    d.NLP = cl_up2(cover < room ? cover : room);
    d.SW = S == 25 ? 5 : 3;
    // [nm, m0, nl, 0], slots int[S][NMP], separable weights double[2 SW][NMP]
    // (wx then wy), node band index, lattice index, owner flag, list length
    // int[NLP] each, entries int[S][NLP], entry weights double[S][NLP]
    d.rank_ints = 4 + S * d.NMP + 4 * d.SW * d.NMP + 4 * d.NLP + 3 * S * d.NLP;
    return d;
}

// Offsets (ints) inside a rank block.
__host__ __device__ inline int clo_mw(const ClusterDims& d) { return 4 + d.S * d.NMP; }
__host__ __device__ inline int clo_nidx(const ClusterDims& d) { return 4 + d.S * d.NMP + 4 * d.SW * d.NMP; }
__host__ __device__ inline int clo_nlat(const ClusterDims& d) { return clo_nidx(d) + d.NLP; }
__host__ __device__ inline int clo_nown(const ClusterDims& d) { return clo_nidx(d) + 2 * d.NLP; }
__host__ __device__ inline int clo_nlen(const ClusterDims& d) { return clo_nidx(d) + 3 * d.NLP; }
__host__ __device__ inline int clo_el(const ClusterDims& d) { return clo_nidx(d) + 4 * d.NLP; }
__host__ __device__ inline int clo_ew(const ClusterDims& d) { return clo_el(d) + d.S * d.NLP; }

inline size_t cluster_plan_ints(int Lb, int S, int C) { return CL_HDR + (size_t)C * cluster_dims(Lb, S, C).rank_ints; }

// Shared memory of the cluster loop: band velocities (x, y) and densities of
// the CTA's nodes, every marker's force (x, y) twice (iteration parity), the
// residual slots twice, and the nodes' lists (entry weights, entry markers).
__host__ __device__ inline size_t cluster_smem_bytes(int Lb, int S, int C)
{
    const ClusterDims d = cluster_dims(Lb, S, C);
    return up16(16 * (size_t)d.NLP) + up16(8 * (size_t)d.NLP) + up16(16 * 2 * (size_t)Lb) + 8 * 2 * 32 +
           up16(8 * (size_t)S * d.NLP) + up16(4 * (size_t)S * d.NLP) + up16(8 * (size_t)S * d.NMP) +
           up16(4 * (size_t)S * d.NMP);
}

// Whether a band step can run on a cluster of C CTAs: one fixed body under MDF
// (its lists cached between steps), the band layout in shared memory, and the
// rank's marker warps plus at least one warp of node threads within one CTA.
inline bool cluster_eligible(const iblbm_ibm_args& a)
{
    const int C = a.cluster_size;
    if (!a.cluster_plan || (C != 2 && C != 4 && C != 8)) return false;
    if (a.method != IBM_MDF || a.mdf_coupled || a.n_particles != 1 || a.xt_table) return false;
    if (a.field_ro || a.field_fstar || a.lb_total < C) return false;
    const int S = a.delta_type == 0 ? 25 : 9;
    const ClusterDims d = cluster_dims(a.lb_total, S, C);
    if (d.MW * 32 + 32 > IBM_THREADS || d.MW * C > 32) return false;
    if ((reinterpret_cast<uintptr_t>(a.cluster_plan) & 7) != 0) return false;
    if (cluster_smem_bytes(a.lb_total, S, C) > (size_t)IBM_SMEM_LIMIT) return false;
    return ibm_smem<double>(a) <= (size_t)IBM_SMEM_LIMIT;  // the layout fits (no global-static form)
}

// ---- distributed shared memory --------------------------------------------------
__device__ __forceinline__ uint32_t cl_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_nranks()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
// The address of the same shared variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cl_map(uint32_t addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cl_store2(uint32_t addr, double x, double y)
{
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(x), "d"(y) : "memory");
}
__device__ __forceinline__ void cl_store_u64(uint32_t addr, unsigned long long v)
{
    asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}
// All threads of all CTAs: prior stores (remote ones included) become visible
// to every CTA's loads after the barrier.
__device__ __forceinline__ void cl_sync()
{
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// Post-streaming moments of lattice node n (the single-CTA step's band_moments, one node).
template <int BC>
__device__ __forceinline__ void cl_node_moments(const iblbm_ibm_args& a, const Geom& g, const BcParams& bc, int n,
                                                double& r, double& x, double& y)
{
    const bool incomp = a.c.incompressible != 0;
    const int j = n / g.nx, i = n - j * g.nx;
    double f[9];
    fstar_node<BC>(a.fpost_prev, a.uring_prev, g, bc, incomp, i, j, f);
    macro_seq(f, incomp, r, x, y);
}

// ---- plan: one CTA per rank, after the band rebuild -----------------------------
template <int A>
__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_cluster_plan_kernel(const iblbm_ibm_args a, int* __restrict__ plan,
                                                                           int C)
{
    constexpr int SW = Sten<A>::SW, S = Sten<A>::S;
    extern __shared__ __align__(16) char smem_raw[];
    int* loc = reinterpret_cast<int*>(smem_raw);  // band index -> local node index (-1: not held)
    int* ired = loc + MAX_BAND;
    const int tid = threadIdx.x, c = blockIdx.x;
    const int Lb = a.lb_total, NB = a.band_capacity;
    const Layout L = make_layout<double>(Lb, NB, S);
    const char* base = reinterpret_cast<const char*>(a.list_cache);
    const int* sidx = reinterpret_cast<const int*>(base + L.o_sidx);
    const int* ent = reinterpret_cast<const int*>(base + L.o_ent);
    const int* cstart = reinterpret_cast<const int*>(base + L.o_cstart);
    const int* nodes = reinterpret_cast<const int*>(base + L.o_nodes);
    const double* wx = reinterpret_cast<const double*>(base + L.o_wx);
    const double* wy = reinterpret_cast<const double*>(base + L.o_wy);
    const double* entw = reinterpret_cast<const double*>(base + L.o_entw);
    const ClusterDims d = cluster_dims(Lb, S, C);
    int* rb = plan + CL_HDR + (size_t)c * d.rank_ints;
    const int nb = *a.band_count;
    const int m0 = (int)((long long)c * Lb / C), m1 = (int)((long long)(c + 1) * Lb / C), nm = m1 - m0;
    int bad = (nb < 1 || nb > NB) ? 1 : 0;
    if (!bad) {
        for (int b = tid; b < nb; b += IBM_THREADS) loc[b] = 0;
        __syncthreads();
        for (int e = tid; e < nm * S; e += IBM_THREADS) loc[sidx[(m0 + e / S) * S + e % S]] = 1;
        __syncthreads();
        // local nodes in band order
        const int ch = (nb + IBM_THREADS - 1) / IBM_THREADS;
        const int b0 = tid * ch, b1 = min(b0 + ch, nb);
        int cnt = 0;
        for (int b = b0; b < b1; ++b) cnt += loc[b];
        int nl;
        int idx = block_exscan(cnt, ired, &nl);
        for (int b = b0; b < b1; ++b) loc[b] = loc[b] ? idx++ : -1;
        __syncthreads();
        if (nl > d.NLP) bad = 1;  // more nodes than the CTA has node threads: the plan does not hold
        for (int b = tid; b < nb && nl <= d.NLP; b += IBM_THREADS) {
            const int i = loc[b];
            if (i < 0) continue;
            const int u0 = cstart[b], n = cstart[b + 1] - u0;
            if (n > S || n < 1) bad = 1;
            const int l0 = ent[u0] >> 5;
            int r0 = 0;
            while (r0 + 1 < C && l0 >= (int)((long long)(r0 + 1) * Lb / C)) ++r0;
            rb[clo_nidx(d) + i] = b;
            rb[clo_nlat(d) + i] = nodes[b];
            rb[clo_nown(d) + i] = r0 == c;
            rb[clo_nlen(d) + i] = min(n, S);
            double* ew = reinterpret_cast<double*>(rb + clo_ew(d));
            for (int j = 0; j < S; ++j) {
                const bool in = j < n;
                rb[clo_el(d) + j * d.NLP + i] = in ? ent[u0 + j] >> 5 : 0;
                ew[j * d.NLP + i] = in ? entw[u0 + j] : 0.0;
            }
        }
        for (int e = tid; e < nm * S; e += IBM_THREADS) {
            const int i = e / S, k = e - i * S, l = m0 + i;
            rb[4 + k * d.NMP + i] = loc[sidx[l * S + k]];
        }
        double* mw = reinterpret_cast<double*>(rb + clo_mw(d));
        for (int e = tid; e < nm * SW; e += IBM_THREADS) {
            const int i = e / SW, q = e - i * SW, l = m0 + i;
            mw[q * d.NMP + i] = wx[l * 5 + q];
            mw[(SW + q) * d.NMP + i] = wy[l * 5 + q];
        }
        if (tid == 0) {
            rb[0] = nm;
            rb[1] = m0;
            rb[2] = nl;
            rb[3] = 0;
        }
    }
    bad = __syncthreads_or(bad);
    if (tid == 0) {
        plan[8 + c] = bad ? 0 : 1;
        if (c == 0) {
            plan[0] = C;
            plan[1] = S;
            plan[2] = Lb;
            plan[3] = nb;
            plan[4] = d.NMP;
            plan[5] = d.NLP;
            plan[6] = 0;
            plan[7] = 0;
        }
    }
}

// ---- the step ---------------------------------------------------------------
template <int A>
__global__ void __launch_bounds__(IBM_THREADS, 1) ibm_cluster_kernel(const iblbm_ibm_args a, BcParams bc,
                                                                      const int* __restrict__ plan)
{
    constexpr int SW = Sten<A>::SW, S = Sten<A>::S;
    extern __shared__ __align__(16) char smem_raw[];
    __shared__ int s_status;
    __shared__ double s_res[2];  // the residual of an iteration (parity)
    const int C = (int)cl_nranks(), rank = (int)cl_rank();
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int Lb = a.lb_total;
    const ClusterDims d = cluster_dims(Lb, S, C);
    const int* rb = plan + CL_HDR + (size_t)rank * d.rank_ints;
    const int MW = d.MW, NSLOT = C * MW, NMP = d.NMP, NLP = d.NLP;
    // this rank's markers, split as the plan splits them
    const int m0 = (int)((long long)rank * Lb / C), nm = (int)((long long)(rank + 1) * Lb / C) - m0;
    const int ni = tid - MW * 32;
    // First round of loads, all independent of one another (the step starts
    // with its plan out of L2): the plan header, this rank's header and each
    // thread's own column of the plan, whatever role the header then confirms.
    int hv[4 + CL_MAX];
#pragma unroll
    for (int r = 0; r < 4; ++r) hv[r] = plan[r];
#pragma unroll
    for (int r = 0; r < CL_MAX; ++r) hv[4 + r] = r < C ? plan[8 + r] : 1;
    const int nb_now = *a.band_count;
    const int nl = rb[2];
    int slot[S];
    double hwx[SW], hwy[SW];
    double dvx = 0, dvy = 0;
    int b = -1, own = 0, len = 0, n = 0;
    if (tid < nm) {
        const double* mw = reinterpret_cast<const double*>(rb + clo_mw(d));
#pragma unroll
        for (int k = 0; k < S; ++k) slot[k] = rb[4 + k * NMP + tid];
#pragma unroll
        for (int q = 0; q < SW; ++q) {
            hwx[q] = mw[q * NMP + tid];
            hwy[q] = mw[(SW + q) * NMP + tid];
        }
        dvx = a.dvel[2 * (m0 + tid)];
        dvy = a.dvel[2 * (m0 + tid) + 1];
    } else if (ni >= 0 && ni < NLP) {
        b = rb[clo_nidx(d) + ni];
        own = rb[clo_nown(d) + ni];
        len = rb[clo_nlen(d) + ni];
        n = rb[clo_nlat(d) + ni];
    }
    // the plan holds iff it was built for this band, these sizes and every rank
    // fits: values every CTA reads alike, so all take the same branch
    int ok = hv[0] == C && hv[1] == S && hv[2] == Lb && hv[3] == nb_now;
#pragma unroll
    for (int r = 0; r < CL_MAX; ++r) ok &= hv[4 + r] == 1;
    if (!ok) {
        if (rank == 0) ibm_step_body<iblbm_ibm_args, double, false, A, IBM_MDF, false, false>(a, bc);
        return;
    }
    const int nls = (nl + 1) & ~1;  // row stride of the entry weights in shared memory
    char* sp = smem_raw;
    double2* s_bw = reinterpret_cast<double2*>(sp);
    sp += up16(16 * (size_t)NLP);
    double* s_bro = reinterpret_cast<double*>(sp);
    sp += up16(8 * (size_t)NLP);
    double2* s_lf = reinterpret_cast<double2*>(sp);
    sp += up16(16 * 2 * (size_t)Lb);
    unsigned long long* s_rb = reinterpret_cast<unsigned long long*>(sp);
    sp += 8 * 2 * 32;
    double* s_ew = reinterpret_cast<double*>(sp);  // entry j of node i: weight s_ew[j * nls + i],
    sp += up16(8 * (size_t)S * NLP);
    int* s_el = reinterpret_cast<int*>(sp);          // marker s_el[j * nls + i]
    sp += up16(4 * (size_t)S * NLP);
    double* s_mw = reinterpret_cast<double*>(sp);    // slot k of marker i: weight s_mw[k * NMP + i],
    sp += up16(8 * (size_t)S * NMP);
    int* s_mi = reinterpret_cast<int*>(sp);          // CTA-local node s_mi[k * NMP + i]
    const Geom g{a.g.nx, a.g.ny, a.g.pitch, a.g.qstride};
    const double dt = a.c.dt;
    const bool unit_dt = (a.c.dt == 1.0);

    // roles: marker threads tid < nm (warps 0 .. MW-1), node threads from MW * 32.
    // A marker's stencil (CTA-local node, weight wx * wy per slot) and a node's
    // list (marker, weight per entry) in shared memory, one column per thread,
    // walked by straight-line code whose loads run ahead of the serial sums.
    const bool mk = tid < nm;
    const bool nd = ni >= 0 && ni < nl;
    const int l = m0 + tid;
    double vs = 0;
    if (mk) {
#pragma unroll
        for (int k = 0; k < S; ++k) {
            s_mi[k * NMP + tid] = slot[k];
            s_mw[k * NMP + tid] = hwx[k / SW] * hwy[k % SW];  // the single-CTA step's wgt(l, k)
        }
        if (a.dvel_scale) {
            const double sc = *a.dvel_scale;
            dvx = dvx * sc;
            dvy = dvy * sc;
        }
    } else if (nd) {
        // second round: the node's list and its post-streaming populations
        const double* ew = reinterpret_cast<const double*>(rb + clo_ew(d));
#pragma unroll
        for (int j = 0; j < S; ++j) {
            const bool in = j < len;
            s_el[j * nls + ni] = in ? rb[clo_el(d) + j * NLP + ni] : 0;
            s_ew[j * nls + ni] = in ? ew[j * NLP + ni] : 0.0;
        }
        double r, x, y;
        switch (a.c.bc) {
        case BC_DIRICHLET_NEUMANN: cl_node_moments<BC_DIRICHLET_NEUMANN>(a, g, bc, n, r, x, y); break;
        case BC_OPEN: cl_node_moments<BC_OPEN>(a, g, bc, n, r, x, y); break;
        case BC_SETTLING: cl_node_moments<BC_SETTLING>(a, g, bc, n, r, x, y); break;
        case BC_TG: cl_node_moments<BC_TG>(a, g, bc, n, r, x, y); break;
        default: cl_node_moments<BC_VELOCITY_INLET>(a, g, bc, n, r, x, y); break;
        }
        s_bro[ni] = r;
        s_bw[ni] = make_double2(x, y);
        vs = dt / (2.0 * r);
    }
    if (tid == 0) {
        s_status = ST_OK;
        if (rank == 0) {
            // exclusion boxes: this step's (checked) and the next step's
            const int x0 = a.box[0], y0 = a.box[1], x1 = a.box[0] + a.box[2] - 1, y1 = a.box[1] + a.box[3] - 1;
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
    }
    // every CTA of the cluster has started (its shared memory may be written)
    // and this CTA's node moments and entry weights are in place
    cl_sync();
    double Rl = 0;
    if (mk) {
        const int* mi = s_mi + tid;
        const double* mwp = s_mw + tid;
#pragma unroll
        for (int k = 0; k < S; ++k) Rl += s_bro[mi[k * NMP]] * mwp[k * NMP];
    }
    const uint32_t lf_base = smem_addr(s_lf), rb_base = smem_addr(s_rb);
    const int min_iter = max(1, min(a.mdf_min_iterations, a.mdf_iterations));
    const double omega = a.mdf_omega;
    double prev = INFINITY, last = INFINITY;
    int iter_count = 0, diverged = 0, converged = 0;
    double lux = 0, luy = 0, lfx = 0, lfy = 0, ftx = 0, fty = 0;
    for (int it = 0; it < a.mdf_iterations; ++it) {
        const int par = it & 1;
        unsigned long long key = 0;  // squared slip as its bit pattern
        if (mk) {
            // slot order; indices and weights from shared memory, the whole
            // stencil unrolled so that its loads issue ahead of the serial sums
            const int* mi = s_mi + tid;
            const double* mwp = s_mw + tid;
            double ux = 0, uy = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const double2 v = s_bw[mi[k * NMP]];
                const double w = mwp[k * NMP];
                ux += v.x * w;
                uy += v.y * w;
            }
            lux = ux;
            luy = uy;
            const double ex = dvx - ux, ey = dvy - uy;
            key = (unsigned long long)__double_as_longlong(ex * ex + ey * ey);
            const double fx = 2.0 * Rl * (dvx - ux), fy = 2.0 * Rl * (dvy - uy);
            lfx = fx;
            lfy = fy;
            if (!unit_dt) {  // x / 1.0 == x: the division only for other time steps
                lfx = fx / dt;
                lfy = fy / dt;
            }
            const uint32_t la = lf_base + (uint32_t)(16 * (par * Lb + l));
            for (int p = 0; p < C; ++p) cl_store2(cl_map(la, (uint32_t)p), lfx, lfy);
        }
        if (wid < MW) {
            const unsigned long long wmax = warp_max_bits(key);
            if (lane == 0) {
                const uint32_t ra = rb_base + (uint32_t)(8 * (par * 32 + rank * MW + wid));
                for (int p = 0; p < C; ++p) cl_store_u64(cl_map(ra, (uint32_t)p), wmax);
            }
        }
        cl_sync();
        // residual = max_l sqrt(slip^2) = sqrt(max_l slip^2), max on the bit patterns:
        // one warp reduces it while the node threads spread (a spread that the
        // divergence check then rejects is undone below)
        if (wid == 0) {
            const double r =
                sqrt(__longlong_as_double((long long)warp_max_bits(lane < NSLOT ? s_rb[par * 32 + lane] : 0ull)));
            if (lane == 0) s_res[par] = r;
        }
        const double ftx0 = ftx, fty0 = fty;
        if (nd) {
            // list order: the first CL_JU entries unrolled (predicated on the
            // list length, so their loads issue together), the rest one by one
            const double2* F = s_lf + par * Lb;
            const int* el = s_el + ni;
            const double* ew = s_ew + ni;
            double ax = 0, ay = 0;
#pragma unroll
            for (int j = 0; j < CL_JU; ++j) {
                if (j < len) {
                    const double2 v = F[el[j * nls]];
                    const double w = ew[j * nls];
                    ax += v.x * w;
                    ay += v.y * w;
                }
            }
            for (int j = CL_JU; j < len; ++j) {
                const double2 v = F[el[j * nls]];
                const double w = ew[j * nls];
                ax += v.x * w;
                ay += v.y * w;
            }
            const double tx = ax * omega, ty = ay * omega;
            ftx += tx;
            fty += ty;
            double2 w = s_bw[ni];
            w.x += tx * vs;
            w.y += ty * vs;
            s_bw[ni] = w;
        }
        __syncthreads();
        const double residual = s_res[par];
        last = residual;
        if (it > 0 && residual > prev * 1.5) {
            // diverged: this iteration's spread is not applied (the working
            // velocities are not read again; the accumulated forces are restored)
            ftx = ftx0;
            fty = fty0;
            diverged = 1;
            iter_count = it + 1;
            break;
        }
        prev = residual;
        iter_count = it + 1;
        if ((it + 1) >= min_iter && residual < a.mdf_tol) {
            converged = 1;
            break;
        }
    }
    if (nd && own) {
        a.band_fib[2 * b] = ftx;
        a.band_fib[2 * b + 1] = fty;
        if (a.band_fib_part) {
            a.band_fib_part[2 * b] = ftx;
            a.band_fib_part[2 * b + 1] = fty;
        }
    }
    if (mk) {
        if (a.Lux) a.Lux[l] = lux;
        if (a.Luy) a.Luy[l] = luy;
        if (a.Lfx) a.Lfx[l] = lfx;
        if (a.Lfy) a.Lfy[l] = lfy;
    }
    if (tid == 0 && rank == 0) {
        a.stats[0] = iter_count;
        a.stats[1] = diverged;
        a.stats[2] = converged;
        a.stats[3] = -3;
        a.dstats[0] = last;
        a.dstats[1] = omega;
        a.stats[4] = s_status;
        if (a.step_counter) *a.step_counter = (*a.step_counter) + 1;
    }
}

// Plan launch (C CTAs, no cluster) after a rebuild.
template <int A>
static int launch_cluster_plan(const iblbm_ibm_args& a, void* stream)
{
    auto K = ibm_cluster_plan_kernel<A>;
    const size_t smem = sizeof(int) * (MAX_BAND + 64);
    if (smem_limit_once<ibm_cluster_plan_kernel<A>>((int)smem) != cudaSuccess) return IBLBM_E_LAUNCH;
    K<<<a.cluster_size, IBM_THREADS, smem, (cudaStream_t)stream>>>(a, a.cluster_plan, a.cluster_size);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

template <int A>
static int launch_cluster_step(const iblbm_ibm_args& a, const BcParams& bc, void* stream)
{
    auto K = ibm_cluster_kernel<A>;
    if (smem_limit_once<ibm_cluster_kernel<A>>(IBM_SMEM_LIMIT) != cudaSuccess) return IBLBM_E_LAUNCH;
    const int S = Sten<A>::S;
    const size_t smem = std::max(ibm_smem<double>(a), cluster_smem_bytes(a.lb_total, S, a.cluster_size));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)a.cluster_size, 1, 1);
    cfg.blockDim = dim3(IBM_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)a.cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int* plan = a.cluster_plan;
    if (cudaLaunchKernelEx(&cfg, K, a, bc, plan) != cudaSuccess) return IBLBM_E_LAUNCH;
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}

}  // namespace iblbm
