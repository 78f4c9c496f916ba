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

// Internal linkage: every class unit instantiates launch_one<YK> for its own
// (class, type), and identical external names would let the linker keep one
// unit's copy for all of them.
namespace {
template <int YK>
cudaError_t launch_one(const LaunchEnv& e, const JKArgs& a0, cudaStream_t st) {
    JKArgs a = a0;
    a.rbuf = jk_rbuf_elems<CX, YK, RT>(e.maxbp[CX], YK >= 0 ? e.maxbp[YK] : 1);
    // K rows in shared memory unless they would not fit (large bases) or
    // the context asks for global rows
    size_t smem = jk_smem_bytes<CX, 1, RT>(e.nao, e.maxbp[CX], a.rbuf, a.kglobal != 0);
    if (!a.kglobal && smem + static_smem((const void*)jk_bra_kernel<CX, 1, RT, YK>) > kSmemLimit) {
        a.kglobal = 1;
        smem = jk_smem_bytes<CX, 1, RT>(e.nao, e.maxbp[CX], a.rbuf, true);
    }
    const void* kernel = (const void*)jk_bra_kernel<CX, 1, RT, YK>;
    cudaError_t r = set_smem_limit(kernel, smem);
    if (r != cudaSuccess) return r;
    a.plan = e.plan_of(CX, YK < 0 ? 0 : YK, sizeof(RT) == sizeof(double) ? 0 : 1);
    jk_bra_kernel<CX, 1, RT, YK><<<persistent_grid(kernel, JK_THREADS, smem, e.nsm), JK_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}
}  // namespace

// split bra classes: one launch per non-empty ket class (largest first), in
// order on st; the others: one launch over all ket classes
cudaError_t AIMD_JK_NAME(const LaunchEnv& e, const JKArgs& a, cudaStream_t st) {
    const int cnt = e.cls_count[CX];
    if (cnt == 0) return cudaSuccess;
    if constexpr (!JKKernel<CX, 1>::SPLIT) {
        return launch_one<-1>(e, a, st);
    } else {
        cudaError_t r = cudaSuccess;
        if constexpr (CX >= 5) if (r == cudaSuccess && e.cls_count[5]) r = launch_one<5>(e, a, st);
        if constexpr (CX >= 4) if (r == cudaSuccess && e.cls_count[4]) r = launch_one<4>(e, a, st);
        if constexpr (CX >= 3) if (r == cudaSuccess && e.cls_count[3]) r = launch_one<3>(e, a, st);
        if constexpr (CX >= 2) if (r == cudaSuccess && e.cls_count[2]) r = launch_one<2>(e, a, st);
        if (r == cudaSuccess && e.cls_count[1]) r = launch_one<1>(e, a, st);
        if (r == cudaSuccess && e.cls_count[0]) r = launch_one<0>(e, a, st);
        return r;
    }
}

}  // namespace hf
