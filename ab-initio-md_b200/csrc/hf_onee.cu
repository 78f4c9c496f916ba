// Launchers of the one-electron kernels (one launch per shell-pair class).
#include "hf_launch.h"

namespace hf {

cudaError_t launch_onee(const LaunchEnv& e, const ShellView& sv, const int* sp_cls_start, const double* origin,
                        double* S, double* T, double* M, double* V, cudaStream_t st, int* nlaunch) {
    const double o[3] = {origin ? origin[0] : 0.0, origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
#define AIMD_LAUNCH_1E(CL)                                                                                   \
    {                                                                                                        \
        const int b0 = sp_cls_start[CL], b1 = sp_cls_start[CL + 1];                                          \
        if (b1 > b0) {                                                                                       \
            onee_kernel<cls_la(CL), cls_lb(CL)><<<(b1 - b0 + 127) / 128, 128, 0, st>>>(sv, b0, b1, o[0], o[1], \
                                                                                      o[2], S, T, M, V); \
            ++*nlaunch;                                                                                      \
        }                                                                                                    \
    }
    AIMD_LAUNCH_1E(0) AIMD_LAUNCH_1E(1) AIMD_LAUNCH_1E(2) AIMD_LAUNCH_1E(3) AIMD_LAUNCH_1E(4) AIMD_LAUNCH_1E(5)
#undef AIMD_LAUNCH_1E
    return cudaGetLastError();
}

cudaError_t launch_onee_grad(const LaunchEnv& e, const ShellView& sv, const int* sp_cls_start, const double* W, const double* D, facc* grad, cudaStream_t st, int* nlaunch) {
    const size_t smem = sizeof(facc) * 3 * e.natm;
    if (smem > 48 * 1024) return cudaErrorInvalidConfiguration;
#define AIMD_LAUNCH_1G(CL)                                                                                    \
    {                                                                                                         \
        const int b0 = sp_cls_start[CL], b1 = sp_cls_start[CL + 1];                                           \
        if (b1 > b0) {                                                                                        \
            onee_grad_kernel<cls_la(CL), cls_lb(CL)><<<(b1 - b0 + 127) / 128, 128, smem, st>>>(sv, b0, b1, W, \
                                                                                              D, grad);      \
            ++*nlaunch;                                                                                       \
        }                                                                                                     \
    }
    AIMD_LAUNCH_1G(0) AIMD_LAUNCH_1G(1) AIMD_LAUNCH_1G(2) AIMD_LAUNCH_1G(3) AIMD_LAUNCH_1G(4) AIMD_LAUNCH_1G(5)
#undef AIMD_LAUNCH_1G
    return cudaGetLastError();
}

}  // namespace hf
