/*
 * aimd_scf: C ABI of the device SCF driver (library libaimd_scf.so, which
 * links libaimd_b200.so, cuBLAS and cuSOLVER). The RHF/UHF DIIS loop of the
 * reference's SCFSolver (Nathan-W123/Ab-Initio-MD, aimd/qc/scf.py:830-923,
 * SCFSolver.run/_iterate) for hosts that are not Python: every matrix stays
 * in device memory, the Fock builds are aimd_jk calls on the same context,
 * the dense algebra is cuBLAS / cuSOLVER on the caller's stream. The host
 * reads two scalars per iteration (energy, commutator norm) and the DIIS
 * Gram row, solves the (m+1)-dimensional Pulay system and decides
 * convergence; the result is a status word, never a trap.
 */
#ifndef AIMD_SCF_H
#define AIMD_SCF_H

#include "aimd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status bits written to *status by aimd_scf_run (the call itself returns
 * an AIMD_* code: AIMD_OK whenever the loop ran). */
#define AIMD_SCF_CONVERGED 1   /* |dE| < conv_energy and max|X^T (FDS - SDF) X| < conv_commutator */
#define AIMD_SCF_MAX_ITER 2    /* max_iter iterations without convergence (last iterate returned) */
#define AIMD_SCF_NONFINITE 4   /* a non-finite energy, commutator or Fock element: stopped there */

/* Options, as the reference's SCFOptions (aimd/qc/scf.py:185-247) where
 * they overlap. RHF: unrestricted = 0 and n_alpha == n_beta. */
typedef struct {
    int n_alpha, n_beta;      /* electrons per spin */
    int unrestricted;         /* 0: RHF (one spin density D/2), 1: UHF (two) */
    int max_iter;             /* default 100 */
    int diis_space;           /* default 8, 0..16; 0 disables DIIS */
    double conv_energy;       /* default 1e-10 Eh */
    double conv_commutator;   /* default 1e-7 */
    double schwarz_threshold; /* default 1e-12 */
    double lindep_threshold;  /* default 1e-7: canonical orthogonalisation below */
    double max_coefficient;   /* default 1e4: larger DIIS coefficients drop the oldest vectors */
} aimd_scf_options;

void aimd_scf_default_options(aimd_scf_options *opt);

/* SCF at the context's current geometry (aimd_set_geometry first).
 *   guess  device [nspin][nao][nao] spin densities (RHF: D/2), or NULL for
 *          the core-Hamiltonian guess;
 *   D, F   device [nspin][nao][nao] outputs: the spin densities of the last
 *          Fock build and that Fock matrix (RHF: one of each);
 *   energy total energy (Eh, nuclear repulsion included) of D; iterations
 *          and status (AIMD_SCF_* bits) on the host.
 * The context's FP32 cutoff (aimd_set_fp32_cutoff) applies to the Fock
 * builds. The driver keeps per-context device workspace between calls;
 * release it with aimd_scf_release before aimd_destroy. */
int aimd_scf_run(aimd_ctx *ctx, const aimd_scf_options *opt, const double *guess, double *D, double *F,
                 double *energy, int *iterations, int *status, void *stream);
int aimd_scf_release(aimd_ctx *ctx);
const char *aimd_scf_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
