// Gradient launcher of one (bra class, ket class) pair (AIMD_KET = 0..AIMD_CLASS) (AIMD_CLASS = 0..5: ss, ps, pp, ds, dp, dd).
#include "hf_launch.h"

#ifndef AIMD_CLASS
#error "compile with -DAIMD_CLASS=<0..5>"
#endif
#define AIMD_CAT2(a, b) a##b
#define AIMD_CAT(a, b) AIMD_CAT2(a, b)

namespace hf {

constexpr int CX = AIMD_CLASS;
using Q0 = QClass<CX, 0>;

#ifndef AIMD_KET
#error "compile with -DAIMD_KET=<0..AIMD_CLASS>"
#endif
constexpr int CY = AIMD_KET;
static_assert(CY <= CX, "ket class above bra class");

cudaError_t AIMD_CAT(AIMD_CAT(AIMD_CAT(launch_grad_c, AIMD_CLASS), _), AIMD_KET)(const LaunchEnv& e, const GradArgs& a,
                                                                                cudaStream_t st) {
    const int cnt = e.cls_count[CX];
    if (cnt == 0 || e.cls_count[CY] == 0) return cudaSuccess;
    const size_t smem = grad_smem_bytes<CX>(e.natm, e.maxbp[CX]);
    cudaError_t r = set_smem_limit((const void*)grad2e_bra_kernel<CX, CY>, smem);
    if (r != cudaSuccess) return r;
    grad2e_bra_kernel<CX, CY><<<cnt, 128, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace hf
