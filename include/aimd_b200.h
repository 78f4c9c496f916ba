/*
 * aimd_b200: C ABI of the B200 (sm_100a) Hartree-Fock integral engine.
 *
 * Plain pointers and sizes only. Device pointers are CUDA device memory of
 * the current device; `stream` is a cudaStream_t (NULL = legacy default
 * stream). Every call returns an AIMD_* status and never traps; on failure
 * aimd_last_error() describes the cause. Calls on one context are not
 * re-entrant (the context holds the geometry-dependent buffers).
 *
 * Each entry point replaces one function of the reference's numba path
 * (Nathan-W123/Ab-Initio-MD, aimd/qc); the reference file:line is given.
 */
#ifndef AIMD_B200_H
#define AIMD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AIMD_ABI_VERSION 1

enum {
    AIMD_OK = 0,
    AIMD_ERR_ARG = 1,          /* null pointer, bad size, no geometry set */
    AIMD_ERR_CUDA = 2,         /* a CUDA call failed (see aimd_last_error) */
    AIMD_ERR_UNSUPPORTED = 3   /* l > 2, or a block with more contractions than the kernel cap */
};

typedef struct aimd_ctx aimd_ctx;

/* Upload one basis (host arrays). Blocks are general-contraction blocks
 * (the reference's BasisSet.blk_*, aimd/qc/basis.py:185-228) with at most
 * 2 contractions for s and 1 otherwise; blk_coef is [nbprim][2], column 1
 * zero for single-contraction blocks. Shells are the segmented shells
 * (BasisSet.shell_*, aimd/qc/basis.py:140-183). All device memory of the
 * engine is allocated here. Replaces the per-geometry setup of
 * aimd/qc/integrals.py:525-627 (_build_pairs) minus the geometry. */
int aimd_create(aimd_ctx **out, int natm, int nao, int nblock, const int *blk_atom, const int *blk_l,
                const int *blk_ncon, const int *blk_ao, const int *blk_p0, const int *blk_np, int nbprim,
                const double *blk_exp, const double *blk_coef, int nshell, const int *sh_atom, const int *sh_l,
                const int *sh_ao, const int *sh_p0, const int *sh_np, int nsprim, const double *sh_exp,
                const double *sh_coef, const double *charges);
int aimd_destroy(aimd_ctx *ctx);

/* New geometry (pos: [natm][3] bohr, host or device): primitive pairs
 * (aimd/qc/integrals.py:525-599 _build_pairs), Schwarz bounds
 * (:864-883 _schwarz_kernel, :970 schwarz_bounds) and the class-sorted
 * pair order used by the quartet lists. */
int aimd_set_geometry(aimd_ctx *ctx, const double *pos, void *stream);

/* Schwarz bounds Q[npair] (device or host pointer), pair index
 * i(i+1)/2 + j over blocks i >= j as in aimd/qc/integrals.py:970. */
int aimd_schwarz(aimd_ctx *ctx, double *Q, void *stream);
int aimd_pair_count(aimd_ctx *ctx);

/* Mixed precision: quartets with Q1 Q2 < cutoff are evaluated in FP32
 * (their contributions still accumulate in FP64, and the Boys function for
 * T >= 40 stays FP64) by aimd_jk, aimd_jk_delta and aimd_grad2e on this
 * context; cutoff 0 (the default) keeps every quartet in FP64. The
 * reference is FP64 throughout; this implements the FP32-below-cutoff rule
 * of the mixed-precision path, applied to the Schwarz product Q1 Q2. */
int aimd_set_fp32_cutoff(aimd_ctx *ctx, double cutoff);

/* Launch shape of the context's J/K and gradient kernels (no counterpart
 * in the reference, whose numba loops have no launch geometry): the work of
 * each class launch is cut into about chunks_per_cta x (resident CTAs)
 * chunks that the persistent CTAs take in turn (1..64, default 8), and a
 * column item of a pair with many primitive quartets is split over bra
 * primitives into items of about item_pq quartets (4..4096, default 32).
 * Results change only by rounding; aimd_b200.engine.Engine.autotune picks
 * the shape by timing. AIMD_ERR_ARG outside the ranges. */
int aimd_set_launch_shape(aimd_ctx *ctx, int chunks_per_cta, int item_pq);
int aimd_get_launch_shape(aimd_ctx *ctx, int *chunks_per_cta, int *item_pq);

/* Integral-direct J/K for nset symmetric densities D[nset][nao][nao]
 * (device). Writes the un-symmetrised accumulators: the caller forms
 * J = J + J^T and K = K + K^T. Quartets with Q1 Q2 < thr are skipped.
 * The K rows of a bra pair's functions are accumulated per CTA in shared
 * memory, or in global memory where they would not fit (large bases; every
 * class when the environment variable AIMD_JK_GLOBAL_K_ROWS=1 is set at
 * aimd_create, a test switch). No size limit on nao from this.
 * Replaces eri_tensor + jk_from_eri (aimd/qc/integrals.py:986-1044). */
int aimd_jk(aimd_ctx *ctx, int nset, const double *D, double *J, double *K, double thr, void *stream);

/* J/K of difference densities D[nset][nao][nao] (device), for incremental
 * Fock builds: quartets with Q1 Q2 < thr are skipped as in aimd_jk, and so
 * are quartets with Q1 Q2 max|D| < dthr, max over the six density blocks
 * the quartet touches (density-weighted Schwarz screening). Same output
 * convention as aimd_jk. No counterpart in the reference, which rebuilds
 * J/K from the full density every iteration (aimd/qc/scf.py:863-867). */
int aimd_jk_delta(aimd_ctx *ctx, int nset, const double *D, double *J, double *K, double thr, double dthr,
                  void *stream);

/* Full screened tensor eri[nao^4] (device), test/debug sizes only. Every
 * quartet is evaluated in FP64 whatever aimd_set_fp32_cutoff set; the
 * context's cutoff is unchanged afterwards.
 * aimd/qc/integrals.py:986-1006 (eri_tensor). */
int aimd_eri_tensor(aimd_ctx *ctx, double *eri, double thr, void *stream);

/* aimd_eri_tensor for callers that may not allocate device memory: the same
 * tensor with the probe scratch (D, J, K of one unit-density Coulomb build)
 * in a static device array of the library instead of cudaMalloc/cudaFree.
 * No counterpart in the reference.
 *   - nao <= AIMD_ERI_STATIC_MAX_NAO (128, 384 KiB of scratch per device);
 *     larger sizes return AIMD_ERR_ARG with a message, before any work;
 *   - every quartet in FP64, as aimd_eri_tensor;
 *   - the context's device must be current; the first call on each device
 *     looks up the scratch address (cudaGetSymbolAddress) and should come
 *     before any stream capture; the address is kept for the life of the
 *     process, so the library must not be used across a cudaDeviceReset of
 *     that device;
 *   - nothing has to be zeroed by the caller; asynchronous on stream (the
 *     tensor is ready when the stream is), unlike aimd_eri_tensor;
 *   - the scratch is one per device: calls that overlap on one device (other
 *     streams, threads or contexts) race and must be serialised by the caller. */
#define AIMD_ERI_STATIC_MAX_NAO 128
int aimd_eri_tensor_static(aimd_ctx *ctx, double *eri, double thr, void *stream);

/* d/dR of 1/2 sum Gamma (mn|ls), Gamma from Dc [nao][nao] and Dx
 * [nx][nao][nao] with exchange factor kfac; grad [natm][3] (device).
 * gamma_bound >= max|Gamma| over all quartets (enumeration bound); the exact
 * per-quartet test is Q1 Q2 max|Gamma| < thr.
 * aimd/qc/integrals.py:1498-1520 (two_electron_gradient). */
int aimd_grad2e(aimd_ctx *ctx, const double *Dc, int nx, const double *Dx, double kfac, double thr,
                double gamma_bound, double *grad, void *stream);

/* S, T, dipole M[3] about origin (host double[3] or NULL) and V, each
 * [nao][nao] (device). aimd/qc/integrals.py:155-329 (_overlap_type_kernel,
 * _nuclear_kernel), :1374-1418. */
int aimd_onee(aimd_ctx *ctx, const double *origin, double *S, double *T, double *M, double *V, void *stream);

/* grad += d/dR [ sum W S + sum D (T + V) ] with W carrying the caller's
 * sign (pass -W for one_electron_gradient). aimd/qc/integrals.py:332-501,
 * :1483-1495. grad must be zeroed by the caller. */
int aimd_onee_grad(aimd_ctx *ctx, const double *W, const double *D, double *grad, void *stream);

/* Inspection: kept quartets per class pair (6 x 6, host), per-pair data. */
int aimd_quartet_counts(aimd_ctx *ctx, int which, int64_t *out_host);
int aimd_pair_data(aimd_ctx *ctx, int *npp_host, int *cls_host, int *sorted_host);

/* Sizes of the context's basis: atoms and AOs. */
int aimd_sizes(aimd_ctx *ctx, int *natm, int *nao);

/* Nuclear repulsion sum_{A<B} Z_A Z_B / R_AB of the current geometry into
 * *energy (host); reads the positions back on `stream` and waits for it.
 * aimd/qc/integrals.py:1421-1426 (nuclear_repulsion_energy). */
int aimd_nuclear_repulsion(aimd_ctx *ctx, double *energy, void *stream);

uint64_t aimd_launch_count(aimd_ctx *ctx);
const char *aimd_last_error(void);
int aimd_version(void);

#ifdef __cplusplus
}
#endif
#endif
