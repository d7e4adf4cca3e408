// ibm_f64.cu — immersed-boundary band step on the FP64 lattice.
//
// The kernel itself is band_kernel.cuh instantiated with R = double; this unit
// is compiled without multiply-add contraction, so every sum runs in the
// reference's order and results are bit-identical to the reference CPU path.
#include <algorithm>
#include <atomic>
#include <mutex>
#include "band_cluster.cuh"

namespace iblbm {
void make_params(const iblbm_case& c, CollParams& cp, BcParams& bc);
}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_ibm_smem_bytes(int lb_total, int band_capacity, int delta_type)
{
    const int S = delta_type == 0 ? 25 : 9;
    return (int)make_layout<double>(lb_total, band_capacity, S).total;
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
    return (int)(make_layout<double>(lb_total, band_capacity, S).static_bytes / sizeof(int));
}

extern "C" int iblbm_ibm_cluster_plan_ints(int lb_total, int delta_type, int cluster_size)
{
    if (lb_total < 1 || (delta_type != 0 && delta_type != 1)) return 0;
    if (cluster_size != 2 && cluster_size != 4 && cluster_size != 8) return 0;
    const int S = delta_type == 0 ? 25 : 9;
    const ClusterDims d = cluster_dims(lb_total, S, cluster_size);
    if (lb_total < cluster_size || d.MW * 32 + 32 > IBM_THREADS || d.MW * cluster_size > 32) return 0;
    if (cluster_smem_bytes(lb_total, S, cluster_size) > (size_t)IBM_SMEM_LIMIT) return 0;
    return (int)cluster_plan_ints(lb_total, S, cluster_size);
}

extern "C" int iblbm_ibm_step_f64(const iblbm_ibm_args* a, void* stream)
{
    const int chk = check_ibm_args<double>(a, true);
    if (chk != IBLBM_OK) return chk;
    CollParams cp;
    BcParams bc;
    make_params(a->c, cp, bc);
    if (cluster_eligible(*a)) {
        if (a->rebuild) {
            // the single-CTA step builds the band and caches its lists; the plan follows from them
            const int rc = dispatch_ibm<iblbm_ibm_args, double, false>(a, bc, stream);
            if (rc != IBLBM_OK) return rc;
            return a->delta_type == 0 ? launch_cluster_plan<2>(*a, stream) : launch_cluster_plan<1>(*a, stream);
        }
        return a->delta_type == 0 ? launch_cluster_step<2>(*a, bc, stream) : launch_cluster_step<1>(*a, bc, stream);
    }
    return dispatch_ibm<iblbm_ibm_args, double, false>(a, bc, stream);
}

// Band steps of n independent cases in one launch (one CTA per case), the
// FP64 counterpart of iblbm_ibm_step_f32_batch: each CTA runs the same band
// step body as the single-case kernel, so every case's results are bit for bit
// those of its own step.
extern "C" int iblbm_ibm_step_f64_batch(const iblbm_ibm_args* host_args, const iblbm_ibm_args* dev_args, int n,
                                        void* stream)
{
    if (!host_args || !dev_args || n < 1 || n > 65535) return IBLBM_E_ARG;
    size_t smem = 0;
    for (int b = 0; b < n; ++b) {
        const int chk = check_ibm_args<double>(&host_args[b]);
        if (chk != IBLBM_OK) return chk;
        smem = std::max(smem, ibm_smem<double>(host_args[b]));
    }
    auto K = ibm_batch_kernel<iblbm_ibm_args, double, false>;
    if (smem_limit_once<ibm_batch_kernel<iblbm_ibm_args, double, false>>(IBM_SMEM_LIMIT) != cudaSuccess) return IBLBM_E_LAUNCH;
    K<<<n, IBM_THREADS, smem, (cudaStream_t)stream>>>(dev_args);
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
// Limits: band_capacity <= 2048 nodes and lb_total <= 1024 markers; larger
// arguments return IBLBM_E_CAPACITY before anything is launched.  The array
// (about 230 KB) lives on every GPU that loads the library until the process
// exits.  All calls share it and it keeps the last call's contents (the kernel
// clears the counters it needs zeroed), so two calls whose kernels overlap on
// the GPU race on it: issue them on one stream, or order them.  The first call
// on each device looks up the array's device address (cudaGetSymbolAddress) with
// that device current; make that first call before any stream capture.  The
// address is kept per device ordinal for the life of the process, which
// assumes the device's primary context does too: after cudaDeviceReset, make
// no further call into this entry point on that device.  The caller still
// passes every input, output and persistent band array.
// ---------------------------------------------------------------------------
namespace iblbm {
constexpr int NOALLOC_MAX_BAND = MAX_BAND;  // the band kernel's own limit (2048)
constexpr int NOALLOC_MAX_MARKERS = 1024;
constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) double g_noalloc_scratch[9 * NOALLOC_MAX_BAND + 9 * NOALLOC_MAX_MARKERS];
static __device__ __align__(256) int g_noalloc_iscratch[NOALLOC_MAX_BAND];
// Device addresses of the two arrays, resolved once per device.  A thread that
// finds no entry resolves both under the lock and publishes the pair with one
// release store, so a reader that sees the pair sees both addresses.
struct NoallocPtrs {
    double* scratch;
    int* iscratch;
};
static NoallocPtrs g_noalloc_store[NOALLOC_MAX_DEVICES];
static std::atomic<const NoallocPtrs*> g_noalloc_ptrs[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_lock;

static const NoallocPtrs* noalloc_ptrs(int dev)
{
    const NoallocPtrs* p = g_noalloc_ptrs[dev].load(std::memory_order_acquire);
    if (p) return p;
    std::lock_guard<std::mutex> hold(g_noalloc_lock);
    p = g_noalloc_ptrs[dev].load(std::memory_order_relaxed);
    if (p) return p;
    void *s = nullptr, *q = nullptr;
    if (cudaGetSymbolAddress(&s, g_noalloc_scratch) != cudaSuccess) return nullptr;
    if (cudaGetSymbolAddress(&q, g_noalloc_iscratch) != cudaSuccess) return nullptr;
    g_noalloc_store[dev] = NoallocPtrs{static_cast<double*>(s), static_cast<int*>(q)};
    g_noalloc_ptrs[dev].store(&g_noalloc_store[dev], std::memory_order_release);
    return &g_noalloc_store[dev];
}
}  // namespace iblbm

extern "C" int iblbm_ibm_step_f64_noalloc(const iblbm_ibm_args* a, void* stream)
{
    if (!a) return IBLBM_E_ARG;
    if (a->band_capacity > NOALLOC_MAX_BAND || a->lb_total > NOALLOC_MAX_MARKERS) return IBLBM_E_CAPACITY;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return IBLBM_E_LAUNCH;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return IBLBM_E_ARG;
    const NoallocPtrs* p = noalloc_ptrs(dev);
    if (!p) return IBLBM_E_LAUNCH;
    iblbm_ibm_args b = *a;
    b.scratch = p->scratch;
    b.iscratch = p->iscratch;
    return iblbm_ibm_step_f64(&b, stream);
}
