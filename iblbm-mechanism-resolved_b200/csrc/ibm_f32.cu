// ibm_f32.cu — immersed-boundary band step on the shifted FP32 lattice.
//
// band_kernel.cuh instantiated with R = float: band moments from g = f - w
// (rho = 1 + sum g), interpolation, spreading and MDF relaxation in FP32, the
// MDF residual norm in FP64; per-marker outputs are written as FP64.
#include <mutex>
#include <algorithm>
#include "band_kernel.cuh"

namespace iblbm {
void make_params32(const iblbm_case& c, CollParams32& cp, BcParams32& bc);
}  // namespace iblbm

using namespace iblbm;

extern "C" int iblbm_ibm32_smem_bytes(int lb_total, int band_capacity, int delta_type)
{
    const int S = delta_type == 0 ? 25 : 9;
    return (int)make_layout<float>(lb_total, band_capacity, S).total;
}

extern "C" int iblbm_ibm32_list_cache_ints(int lb_total, int band_capacity, int delta_type)
{
    const int S = delta_type == 0 ? 25 : 9;
    return (int)(make_layout<float>(lb_total, band_capacity, S).static_bytes / sizeof(int));
}

extern "C" int iblbm_ibm_step_f32(const iblbm_ibm32_args* a, void* stream)
{
    const int chk = check_ibm_args<float>(a, true);
    if (chk != IBLBM_OK) return chk;
    CollParams32 cp;
    BcParams32 bc;
    make_params32(a->c, cp, bc);
    return dispatch_ibm<iblbm_ibm32_args, float, true>(a, bc, stream);
}

extern "C" int iblbm_ibm_step_f32_batch(const iblbm_ibm32_args* host_args, const iblbm_ibm32_args* dev_args, int n,
                                        void* stream)
{
    if (!host_args || !dev_args || n < 1 || n > 65535) return IBLBM_E_ARG;
    size_t smem = 0;
    for (int b = 0; b < n; ++b) {
        const int chk = check_ibm_args<float>(&host_args[b]);
        if (chk != IBLBM_OK) return chk;
        smem = std::max(smem, ibm_smem<float>(host_args[b]));
    }
    auto K = ibm_batch_kernel<iblbm_ibm32_args, float, true>;
    if (smem_limit_once<ibm_batch_kernel<iblbm_ibm32_args, float, true>>(IBM_SMEM_LIMIT) != cudaSuccess) return IBLBM_E_LAUNCH;
    K<<<n, IBM_THREADS, smem, (cudaStream_t)stream>>>(dev_args);
    return cudaGetLastError() == cudaSuccess ? IBLBM_OK : IBLBM_E_LAUNCH;
}
