// Gradient launcher of one (bra class, ket class) pair (AIMD_CLASS = 0..5: ss, ps, pp, ds, dp, dd;
// AIMD_KET = 0..AIMD_CLASS) and one arithmetic type (AIMD_REAL = 0: FP64; 1: FP32 quartets of the
// mixed-precision path).
#include "hf_launch.h"

#ifndef AIMD_CLASS
#error "compile with -DAIMD_CLASS=<0..5>"
#endif
#ifndef AIMD_KET
#error "compile with -DAIMD_KET=<0..AIMD_CLASS>"
#endif
#ifndef AIMD_REAL
#define AIMD_REAL 0
#endif
#define AIMD_CAT2(a, b) a##b
#define AIMD_CAT(a, b) AIMD_CAT2(a, b)

namespace hf {

constexpr int CX = AIMD_CLASS;
constexpr int CY = AIMD_KET;
static_assert(CY <= CX, "ket class above bra class");

#if AIMD_REAL == 0
using RT = double;
#define AIMD_GRAD_NAME AIMD_CAT(AIMD_CAT(AIMD_CAT(launch_grad_c, AIMD_CLASS), _), AIMD_KET)
#else
using RT = float;
#define AIMD_GRAD_NAME AIMD_CAT(AIMD_CAT(AIMD_CAT(launch_grad32_c, AIMD_CLASS), _), AIMD_KET)
#endif

cudaError_t AIMD_GRAD_NAME(const LaunchEnv& e, const GradArgs& a0, cudaStream_t st) {
    const int cnt = e.cls_count[CX];
    if (cnt == 0 || e.cls_count[CY] == 0) return cudaSuccess;
    GradArgs a = a0;
    a.rbuf = grad_rbuf_elems<CX, CY, RT>(e.maxbp[CX], e.maxbp[CY]);
    const size_t smem = grad_smem_bytes<CX, RT>(e.natm, e.maxbp[CX], a.rbuf);
    const void* kernel = (const void*)grad2e_bra_kernel<CX, CY, RT>;
    cudaError_t r = set_smem_limit(kernel, smem);
    if (r != cudaSuccess) return r;
    a.plan = e.plan_of(CX, CY, sizeof(RT) == sizeof(double) ? 0 : 1);
    grad2e_bra_kernel<CX, CY, RT><<<persistent_grid(kernel, GRAD_THREADS, smem, e.nsm), GRAD_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace hf
