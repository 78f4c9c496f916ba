// Host-side launchers of the class-templated kernels. Each bra pair class
// lives in its own translation units (hf_class_jk.cu compiled with
// -DAIMD_CLASS=0..5, hf_class_grad.cu with -DAIMD_CLASS=X -DAIMD_KET=Y for
// Y <= X), once per arithmetic type (-DAIMD_REAL=0: FP64, the launchers
// below without a suffix; -DAIMD_REAL=1: the FP32 quartets of the
// mixed-precision path, suffix 32), so that they compile in parallel.
// Gradient launchers with Y > X are declared but never defined or called.
#pragma once
#include <cuda_runtime.h>

#include "hf_grad.cuh"
#include "hf_onee.cuh"

namespace hf {

struct LaunchEnv {
    int cls_count[NCLS];     // block pairs per class
    int cls_start[NCLS + 1]; // start of each class in the class-grouped order
    int maxbp[NCLS];         // largest primitive-pair count of a block pair, per class
    int nao, natm;
    const int* by_class;     // pair indices grouped by class
    double* Q;
    int nsm;                 // SMs of the device
    // work plans of the class kernels: per (type, ket class) one [npair +
    // NCLS] array holding the [nbra + 1] prefix of each bra class in turn;
    // chunk counters per (type, bra class, ket class)
    int* plan;
    int* plan_next;
    int plan_stride;
    WorkPlan plan_of(int cx, int cy, int rt) const {
        return WorkPlan{plan + (size_t)(rt * NCLS + cy) * plan_stride + cls_start[cx] + cx,
                        plan_next + (rt * NCLS + cx) * NCLS + cy};
    }
};

// CTAs of a persistent launch of `kernel`: as many as fit on the device.
inline int persistent_grid(const void* kernel, int threads, size_t smem, int nsm) {
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) per = 1;
    return per * nsm;
}

// Status: cudaSuccess, a CUDA error, or cudaErrorInvalidConfiguration when
// the shared-memory request exceeds the per-CTA limit.
#define AIMD_DECLARE_TYPED(X, S)                                                                       \
    cudaError_t launch_jk##S##_c##X(const LaunchEnv& e, const JKArgs& a, cudaStream_t st);              \
    cudaError_t launch_grad##S##_c##X##_0(const LaunchEnv& e, const GradArgs& a, cudaStream_t st);     \
    cudaError_t launch_grad##S##_c##X##_1(const LaunchEnv& e, const GradArgs& a, cudaStream_t st);     \
    cudaError_t launch_grad##S##_c##X##_2(const LaunchEnv& e, const GradArgs& a, cudaStream_t st);     \
    cudaError_t launch_grad##S##_c##X##_3(const LaunchEnv& e, const GradArgs& a, cudaStream_t st);     \
    cudaError_t launch_grad##S##_c##X##_4(const LaunchEnv& e, const GradArgs& a, cudaStream_t st);     \
    cudaError_t launch_grad##S##_c##X##_5(const LaunchEnv& e, const GradArgs& a, cudaStream_t st);
#define AIMD_DECLARE_CLASS(X)                                                                          \
    cudaError_t launch_schwarz_c##X(const LaunchEnv& e, const QuartetArgs& q, cudaStream_t st);         \
    AIMD_DECLARE_TYPED(X, )                                                                            \
    AIMD_DECLARE_TYPED(X, 32)
AIMD_DECLARE_CLASS(0)
AIMD_DECLARE_CLASS(1)
AIMD_DECLARE_CLASS(2)
AIMD_DECLARE_CLASS(3)
AIMD_DECLARE_CLASS(4)
AIMD_DECLARE_CLASS(5)
#undef AIMD_DECLARE_CLASS
#undef AIMD_DECLARE_TYPED

cudaError_t launch_onee(const LaunchEnv& e, const ShellView& sv, const int* sp_cls_start, const double* origin,
                        double* S, double* T, double* M, double* V, cudaStream_t st, int* nlaunch);
cudaError_t launch_onee_grad(const LaunchEnv& e, const ShellView& sv, const int* sp_cls_start, const double* W,
                             const double* D, facc* grad, cudaStream_t st, int* nlaunch);

constexpr size_t kSmemLimit = 227 * 1024;     // dynamic shared memory per CTA (sm_100a)

// Allow `bytes` of dynamic shared memory for `kernel`. The default limit is
// 48 KB for static plus dynamic shared memory together, so the opt-in is
// needed whenever the sum passes it; the sum may not pass kSmemLimit. The
// attribute is per kernel and process-wide, and contexts of different
// bases run the same kernels from several host threads at once (batched
// geometries), so it is always raised to the whole per-CTA limit, never
// set to one launch's need: a smaller value set by one thread would make
// another thread's larger launch fail.
inline cudaError_t set_smem_limit(const void* kernel, size_t bytes) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    if (bytes + fa.sharedSizeBytes > kSmemLimit) return cudaErrorInvalidConfiguration;
    if (bytes + fa.sharedSizeBytes > 48 * 1024 &&
        (size_t)fa.maxDynamicSharedSizeBytes + fa.sharedSizeBytes < kSmemLimit)
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kSmemLimit - fa.sharedSizeBytes));
    return cudaSuccess;
}

// Static shared memory of `kernel` (0 if the query fails).
inline size_t static_smem(const void* kernel) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kernel) == cudaSuccess ? fa.sharedSizeBytes : 0;
}

}  // namespace hf
