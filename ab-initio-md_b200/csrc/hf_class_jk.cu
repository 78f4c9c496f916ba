// J/K and Schwarz launchers of one bra pair class (AIMD_CLASS = 0..5: ss, ps, pp, ds, dp, dd) and one
// arithmetic type (AIMD_REAL = 0: FP64 J/K + Schwarz; 1: FP32 J/K quartets of the mixed-precision path).
#include "hf_launch.h"

#ifndef AIMD_CLASS
#error "compile with -DAIMD_CLASS=<0..5>"
#endif
#ifndef AIMD_REAL
#define AIMD_REAL 0
#endif
#define AIMD_CAT2(a, b) a##b
#define AIMD_CAT(a, b) AIMD_CAT2(a, b)

namespace hf {

constexpr int CX = AIMD_CLASS;
using Q0 = QClass<CX, 0>;

#if AIMD_REAL == 0
using RT = double;
#define AIMD_JK_NAME AIMD_CAT(launch_jk_c, AIMD_CLASS)

cudaError_t AIMD_CAT(launch_schwarz_c, AIMD_CLASS)(const LaunchEnv& e, const QuartetArgs& q, cudaStream_t st) {
    const int cnt = e.cls_count[CX];
    if (cnt == 0) return cudaSuccess;
    const size_t smem = sizeof(double) * (size_t)e.maxbp[CX] * (BraE<Q0::LA, Q0::LB, 0>::SIZE + SBW);
    cudaError_t r = set_smem_limit((const void*)schwarz_kernel<CX>, smem);
    if (r != cudaSuccess) return r;
    schwarz_kernel<CX><<<cnt, 64, smem, st>>>(q, e.by_class + e.cls_start[CX], e.Q);
    return cudaGetLastError();
}
#else
using RT = float;
#define AIMD_JK_NAME AIMD_CAT(launch_jk32_c, AIMD_CLASS)
#endif

cudaError_t AIMD_JK_NAME(const LaunchEnv& e, const JKArgs& a, cudaStream_t st) {
    const int cnt = e.cls_count[CX];
    if (cnt == 0) return cudaSuccess;
    const size_t smem = jk_smem_bytes<CX, 1, RT>(e.nao, e.maxbp[CX]);
    cudaError_t r = set_smem_limit((const void*)jk_bra_kernel<CX, 1, RT>, smem);
    if (r != cudaSuccess) return r;
    jk_bra_kernel<CX, 1, RT><<<cnt * JKKernel<CX, 1>::NY, JK_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace hf
