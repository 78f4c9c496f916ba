// Device SCF driver behind the C ABI (library libaimd_scf.so, linked against
// libaimd_b200.so, cuBLAS and cuSOLVER): the RHF/UHF DIIS loop of the
// reference's SCFSolver (aimd/qc/scf.py:869-923) for hosts that are not
// Python. Every matrix stays on the device; per iteration the host reads two
// scalars (the energy and the commutator norm) to decide convergence, and
// the small DIIS system ((m+1) x (m+1), m <= diis_space).
//
//   F_s = h + g sum_t J[D_t] - K[D_s]   (g = 2 RHF, 1 UHF), symmetrised
//   E   = E_nn + g/2 sum_s tr D_s (h + F_s)
//   e_s = X^T (F_s D_s S - S D_s F_s) X,  converged when |dE| < conv_energy
//         and max|e| < conv_commutator
//   DIIS on (X^T F X, e) with the Pulay equations, eigh of X^T F X, aufbau.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/aimd_scf.h"

namespace {

thread_local char g_scf_err[512] = "";

#define SCF_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            snprintf(g_scf_err, sizeof g_scf_err, "%s: %s", #call, cudaGetErrorString(e_));     \
            return AIMD_ERR_CUDA;                                                               \
        }                                                                                       \
    } while (0)
#define SCF_LIB(call, what)                                                                     \
    do {                                                                                        \
        if ((call) != 0) {                                                                      \
            snprintf(g_scf_err, sizeof g_scf_err, "%s failed", what);                           \
            return AIMD_ERR_CUDA;                                                               \
        }                                                                                       \
    } while (0)
#define SCF_ABI(call, what)                                                                     \
    do {                                                                                        \
        int r_ = (call);                                                                        \
        if (r_ != AIMD_OK) {                                                                    \
            snprintf(g_scf_err, sizeof g_scf_err, "%s: %s", what, aimd_last_error());           \
            return r_;                                                                          \
        }                                                                                       \
    } while (0)

// out[i][j] = 0.5 (a[i][j] + a[j][i]) for nmat n x n matrices (out may be a)
__global__ void symmetrize_kernel(int n, int nmat, const double* a, double* out) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)nmat * n * n) return;
    const long m = i / ((long)n * n), r = (i / n) % n, c = i % n;
    if (c < r) return;
    const double* A = a + m * n * n;
    const double v = 0.5 * (A[r * n + c] + A[c * n + r]);
    out[m * n * n + r * n + c] = v;
    out[m * n * n + c * n + r] = v;
}

// F_s = h + g sum_t J_t - K_s with J = Ja + Ja^T, K = Ka + Ka^T built from
// the un-symmetrised accumulators of aimd_jk (symmetric by construction)
__global__ void fock_kernel(int n, int nspin, double g, const double* H, const double* Ja, const double* Ka,
                            double* F) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nn = (long)n * n;
    if (i >= nn) return;
    const long t = (i % n) * n + i / n;
    double j = 0.0;
    for (int s = 0; s < nspin; ++s) j += Ja[s * nn + i] + Ja[s * nn + t];
    for (int s = 0; s < nspin; ++s) F[s * nn + i] = H[i] + g * j - (Ka[s * nn + i] + Ka[s * nn + t]);
}

// energy and commutator norm: out[0] = sum_s tr D_s (h + F_s), out[1] = max|e|
__global__ void reduce_kernel(long nn, int nspin, const double* D, const double* H, const double* F, long ne,
                              const double* err, double* out) {
    __shared__ double se[256], sm[256];
    double e = 0.0, m = 0.0;
    for (long i = threadIdx.x; i < nn * nspin; i += blockDim.x) {
        const long s = i / nn, k = i % nn;
        e += D[i] * (H[k] + F[s * nn + k]);
    }
    for (long i = threadIdx.x; i < ne; i += blockDim.x) m = fmax(m, fabs(err[i]));
    se[threadIdx.x] = e;
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            se[threadIdx.x] += se[threadIdx.x + w];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = se[0];
        out[1] = sm[0];
    }
}

// y = sum_i c_i x_i for m vectors of length len (c on the device)
__global__ void combine_kernel(long len, int m, const double* const* x, const double* c, double* y) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= len) return;
    double v = 0.0;
    for (int k = 0; k < m; ++k) v += c[k] * x[k][i];
    y[i] = v;
}

inline int blocks(long n) { return (int)((n + 255) / 256); }

// Per-context workspace of the driver, kept between calls.
struct Work {
    aimd_ctx* ctx = nullptr;
    int n = 0, nspin = 0, space = 0, nmo = 0;
    double *S = nullptr, *T = nullptr, *M = nullptr, *V = nullptr, *H = nullptr, *X = nullptr;
    double *Ja = nullptr, *Ka = nullptr, *F = nullptr, *Dn = nullptr, *t1 = nullptr, *t2 = nullptr, *err = nullptr;
    double *Fo = nullptr, *w = nullptr, *solver_ws = nullptr, *red = nullptr, *coef = nullptr;
    double *hist_f = nullptr, *hist_e = nullptr;   // [space][nspin][nmo][nmo]
    double **ptrs = nullptr;
    int* info = nullptr;
    int lwork = 0;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t sol = nullptr;
};

void release(Work& w) {
    void* p[] = {w.S, w.T, w.M, w.V, w.H, w.X, w.Ja, w.Ka, w.F, w.Dn, w.t1, w.t2, w.err, w.Fo, w.w, w.solver_ws,
                 w.red, w.coef, w.hist_f, w.hist_e, w.ptrs, w.info};
    for (void* q : p) cudaFree(q);
    if (w.blas) cublasDestroy(w.blas);
    if (w.sol) cusolverDnDestroy(w.sol);
    w = Work();
}

// Pulay DIIS: minimise |sum c_i e_i| subject to sum c_i = 1 from the Gram
// matrix B_ij = <e_i, e_j> (host, m <= 16), by Gaussian elimination with
// partial pivoting of the bordered system. Returns false if singular.
bool pulay(int m, const double* B, double* c) {
    const int k = m + 1;
    std::vector<double> A((size_t)k * (k + 1), 0.0);
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(B[i * m + i]));
    if (!(scale > 0.0)) return false;
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) A[i * (k + 1) + j] = B[i * m + j] / scale;
        A[i * (k + 1) + m] = -1.0;
        A[m * (k + 1) + i] = -1.0;
    }
    A[m * (k + 1) + k] = -1.0;                  // right-hand side (0, ..., 0, -1)
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int r = col + 1; r < k; ++r)
            if (fabs(A[r * (k + 1) + col]) > fabs(A[piv * (k + 1) + col])) piv = r;
        if (fabs(A[piv * (k + 1) + col]) < 1e-300) return false;
        if (piv != col)
            for (int j = 0; j <= k; ++j) std::swap(A[col * (k + 1) + j], A[piv * (k + 1) + j]);
        for (int r = 0; r < k; ++r) {
            if (r == col) continue;
            const double f = A[r * (k + 1) + col] / A[col * (k + 1) + col];
            for (int j = col; j <= k; ++j) A[r * (k + 1) + j] -= f * A[col * (k + 1) + j];
        }
    }
    for (int i = 0; i < m; ++i) {
        c[i] = A[i * (k + 1) + k] / A[i * (k + 1) + i];
        if (!std::isfinite(c[i])) return false;
    }
    return true;
}

}  // namespace

extern "C" const char* aimd_scf_last_error(void) { return g_scf_err; }

extern "C" void aimd_scf_default_options(aimd_scf_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->max_iter = 100;
    o->diis_space = 8;
    o->conv_energy = 1e-10;
    o->conv_commutator = 1e-7;
    o->schwarz_threshold = 1e-12;
    o->lindep_threshold = 1e-7;
    o->max_coefficient = 1e4;
}

namespace {

// X (column-major n x nmo) from eigh(S): symmetric S^-1/2 when every
// eigenvalue reaches the threshold, else canonical U_keep s_keep^-1/2
// (aimd/qc/scf.py:284-303, "auto").
__global__ void scale_columns_kernel(int n, int ncol, int off, const double* U, const double* w, double* out) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)n * ncol) return;
    const long r = i % n, c = i / n;
    out[i] = U[(c + off) * (long)n + r] / sqrt(w[c + off]);
}

__global__ void add_kernel(long len, const double* a, const double* b, double* out) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < len) out[i] = a[i] + b[i];
}

__global__ void is_finite_kernel(long len, const double* a, int* flag) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < len && !isfinite(a[i])) *flag = 1;
}

Work* work_for(aimd_ctx* ctx, int n, int nspin, int space) {
    static std::vector<Work> pool;
    for (Work& w : pool)
        if (w.ctx == ctx) {
            if (w.n == n && w.nspin == nspin && w.space == space) return &w;
            release(w);
            w.ctx = ctx;
            return &w;
        }
    pool.emplace_back();
    pool.back().ctx = ctx;
    return &pool.back();
}

int setup(Work& w, int n, int nspin, int space) {
    if (w.S) return AIMD_OK;
    w.n = n;
    w.nspin = nspin;
    w.space = space;
    const size_t nn = (size_t)n * n;
    auto al = [](double** p, size_t cnt) { return cudaMalloc(reinterpret_cast<void**>(p), (cnt ? cnt : 1) * sizeof(double)); };
    SCF_CUDA(al(&w.S, nn)); SCF_CUDA(al(&w.T, nn)); SCF_CUDA(al(&w.M, 3 * nn)); SCF_CUDA(al(&w.V, nn));
    SCF_CUDA(al(&w.H, nn)); SCF_CUDA(al(&w.X, nn)); SCF_CUDA(al(&w.Ja, 2 * nn)); SCF_CUDA(al(&w.Ka, 2 * nn));
    SCF_CUDA(al(&w.F, 2 * nn)); SCF_CUDA(al(&w.Dn, 2 * nn)); SCF_CUDA(al(&w.t1, nn)); SCF_CUDA(al(&w.t2, nn));
    SCF_CUDA(al(&w.err, 2 * nn)); SCF_CUDA(al(&w.Fo, 2 * nn)); SCF_CUDA(al(&w.w, n)); SCF_CUDA(al(&w.red, 4 + 64));
    SCF_CUDA(al(&w.coef, 64));
    SCF_CUDA(al(&w.hist_f, (size_t)(space > 0 ? space : 1) * 2 * nn));
    SCF_CUDA(al(&w.hist_e, (size_t)(space > 0 ? space : 1) * 2 * nn));
    SCF_CUDA(cudaMalloc(reinterpret_cast<void**>(&w.ptrs), 64 * sizeof(double*)));
    SCF_CUDA(cudaMalloc(reinterpret_cast<void**>(&w.info), 4 * sizeof(int)));
    SCF_LIB(cublasCreate(&w.blas), "cublasCreate");
    SCF_LIB(cusolverDnCreate(&w.sol), "cusolverDnCreate");
    SCF_LIB(cusolverDnDsyevd_bufferSize(w.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, w.t1, n, w.w,
                                        &w.lwork), "cusolverDnDsyevd_bufferSize");
    SCF_CUDA(al(&w.solver_ws, (size_t)w.lwork));
    return AIMD_OK;
}

// eigenvalues (ascending) into w.w and vectors (columns) in A, m x m in place
int eigh(Work& w, double* A, int m) {
    SCF_LIB(cusolverDnDsyevd(w.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, A, m, w.w, w.solver_ws,
                             w.lwork, w.info), "cusolverDnDsyevd");
    return AIMD_OK;
}

// D_s = C C^T with C = X Cp[:, :nocc] (the nocc lowest orbitals of Fo_s = Cp diag Cp^T)
int aufbau(Work& w, double* Fo_s, int nocc, double* D_s, cudaStream_t st) {
    const int n = w.n, m = w.nmo;
    const double one = 1.0, zero = 0.0;
    if (int r = eigh(w, Fo_s, m)) return r;
    if (nocc == 0) {
        SCF_CUDA(cudaMemsetAsync(D_s, 0, sizeof(double) * n * n, st));
        return AIMD_OK;
    }
    // C (n x nocc) = X (n x m) Cp[:, :nocc] (m x nocc)
    SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, nocc, m, &one, w.X, n, Fo_s, m, &zero, w.t1, n),
            "cublasDgemm C");
    SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_T, n, n, nocc, &one, w.t1, n, w.t1, n, &zero, D_s, n),
            "cublasDgemm D");
    return AIMD_OK;
}

}  // namespace

extern "C" int aimd_scf_run(aimd_ctx* ctx, const aimd_scf_options* opt, const double* guess, double* D, double* F,
                            double* energy, int* iterations, int* status, void* stream) {
    if (!ctx || !opt || !D || !F || !energy || !iterations || !status) {
        snprintf(g_scf_err, sizeof g_scf_err, "aimd_scf_run: null argument");
        return AIMD_ERR_ARG;
    }
    *status = 0;
    *iterations = 0;
    int natm = 0, n = 0;
    SCF_ABI(aimd_sizes(ctx, &natm, &n), "aimd_sizes");
    const int nspin = opt->unrestricted ? 2 : 1;
    const int na = opt->n_alpha, nb = opt->n_beta;
    if (na < 0 || nb < 0 || nb > na || na > n || (!opt->unrestricted && na != nb) || opt->max_iter < 1 ||
        opt->diis_space < 0 || opt->diis_space > 16 || !(opt->conv_energy > 0.0) || !(opt->conv_commutator > 0.0)) {
        snprintf(g_scf_err, sizeof g_scf_err, "aimd_scf_run: invalid options (electrons %d/%d for %d AOs, "
                 "max_iter %d, diis_space %d in 0..16, positive thresholds)", na, nb, n, opt->max_iter,
                 opt->diis_space);
        return AIMD_ERR_ARG;
    }
    const int nocc[2] = {na, nb};
    const double g = 2.0 / nspin;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Work* wp = work_for(ctx, n, nspin, opt->diis_space);
    if (int r = setup(*wp, n, nspin, opt->diis_space)) return r;
    Work& w = *wp;
    const size_t nn = (size_t)n * n;
    const double one = 1.0, zero = 0.0, mone = -1.0;
    SCF_LIB(cublasSetStream(w.blas, st), "cublasSetStream");
    SCF_LIB(cusolverDnSetStream(w.sol, st), "cusolverDnSetStream");
    double enuc = 0.0;
    SCF_ABI(aimd_nuclear_repulsion(ctx, &enuc, stream), "aimd_nuclear_repulsion");

    // one-electron matrices, h = T + V (symmetrised), X from eigh(S)
    SCF_ABI(aimd_onee(ctx, nullptr, w.S, w.T, w.M, w.V, stream), "aimd_onee");
    add_kernel<<<blocks(nn), 256, 0, st>>>(nn, w.T, w.V, w.H);
    symmetrize_kernel<<<blocks(nn), 256, 0, st>>>(n, 1, w.H, w.H);
    SCF_CUDA(cudaMemcpyAsync(w.t2, w.S, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    if (int r = eigh(w, w.t2, n)) return r;
    std::vector<double> s(n);
    SCF_CUDA(cudaMemcpyAsync(s.data(), w.w, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    SCF_CUDA(cudaStreamSynchronize(st));
    int off = 0;
    while (off < n && s[off] < opt->lindep_threshold) ++off;
    if (off == n) {
        snprintf(g_scf_err, sizeof g_scf_err, "aimd_scf_run: every overlap eigenvalue is below lindep_threshold");
        return AIMD_ERR_ARG;
    }
    w.nmo = n - off;
    if (nocc[0] > w.nmo) {
        snprintf(g_scf_err, sizeof g_scf_err, "aimd_scf_run: %d electrons of one spin in %d orbitals", nocc[0],
                 w.nmo);
        return AIMD_ERR_ARG;
    }
    const int m = w.nmo;
    if (off == 0) {
        // X = U s^-1/2 U^T
        scale_columns_kernel<<<blocks(nn), 256, 0, st>>>(n, n, 0, w.t2, w.w, w.t1);
        SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_T, n, n, n, &one, w.t1, n, w.t2, n, &zero, w.X, n),
                "cublasDgemm X");
    } else {
        scale_columns_kernel<<<blocks((long)n * m), 256, 0, st>>>(n, m, off, w.t2, w.w, w.X);
    }
    SCF_CUDA(cudaGetLastError());
    // Fo_s = X^T A X (m x m) of a symmetric n x n matrix A
    auto transform = [&](const double* A, double* out) -> int {
        SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, &one, A, n, w.X, n, &zero, w.t1, n), "AX");
        SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, &one, w.X, n, w.t1, n, &zero, out, m), "XtAX");
        return AIMD_OK;
    };
    // initial spin densities: the caller's guess (symmetrised), or the core Hamiltonian's orbitals
    if (guess) {
        symmetrize_kernel<<<blocks(nspin * nn), 256, 0, st>>>(n, nspin, guess, D);
        SCF_CUDA(cudaGetLastError());
    } else {
        for (int sp = 0; sp < nspin; ++sp) {
            if (int r = transform(w.H, w.Fo)) return r;
            if (int r = aufbau(w, w.Fo, nocc[sp], D + sp * nn, st)) return r;
        }
    }

    const int space = opt->diis_space;
    std::vector<double> gram((size_t)space * space, 0.0), c(space > 0 ? space : 1);
    std::vector<int> slot_age;                      // history slots, oldest first
    double e_prev = NAN, best = INFINITY;
    int since_best = 0;
    const long ne = (long)nspin * m * m;
    double host[2] = {0.0, 0.0};
    int conv = 0, it = 0;
    for (it = 1; it <= opt->max_iter; ++it) {
        SCF_ABI(aimd_jk(ctx, nspin, D, w.Ja, w.Ka, opt->schwarz_threshold, stream), "aimd_jk");
        fock_kernel<<<blocks(nn), 256, 0, st>>>(n, nspin, g, w.H, w.Ja, w.Ka, F);
        SCF_CUDA(cudaGetLastError());
        // e_s = X^T (F D S - S D F) X; F, D, S symmetric, so S D F = (F D S)^T
        for (int sp = 0; sp < nspin; ++sp) {
            const double* Fs = F + sp * nn;
            const double* Ds = D + sp * nn;
            SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, Fs, n, Ds, n, &zero, w.t1, n), "FD");
            SCF_LIB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, w.t1, n, w.S, n, &zero, w.t2, n),
                    "FDS");
            SCF_LIB(cublasDgeam(w.blas, CUBLAS_OP_N, CUBLAS_OP_T, n, n, &one, w.t2, n, &mone, w.t2, n, w.t1, n),
                    "FDS-SDF");
            if (int r = transform(w.t1, w.err + (size_t)sp * m * m)) return r;
        }
        reduce_kernel<<<1, 256, 0, st>>>(nn, nspin, D, w.H, F, ne, w.err, w.red);
        SCF_CUDA(cudaMemsetAsync(w.info + 1, 0, sizeof(int), st));
        is_finite_kernel<<<blocks(nspin * nn), 256, 0, st>>>(nspin * nn, F, w.info + 1);
        SCF_CUDA(cudaGetLastError());
        int nonfinite = 0;
        SCF_CUDA(cudaMemcpyAsync(host, w.red, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        SCF_CUDA(cudaMemcpyAsync(&nonfinite, w.info + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCF_CUDA(cudaStreamSynchronize(st));
        const double e_el = 0.5 * g * host[0], err_norm = host[1];
        *energy = e_el + enuc;
        if (nonfinite || !std::isfinite(e_el) || !std::isfinite(err_norm)) {
            *status = AIMD_SCF_NONFINITE;
            *iterations = it;
            return AIMD_OK;
        }
        const double de = e_el - e_prev;
        if (std::fabs(de) < opt->conv_energy && err_norm < opt->conv_commutator) {
            conv = 1;
            break;
        }
        if (it == opt->max_iter) break;
        // Fo = X^T F X, DIIS extrapolation over the stored (Fo, e) pairs
        for (int sp = 0; sp < nspin; ++sp)
            if (int r = transform(F + sp * nn, w.Fo + (size_t)sp * m * m)) return r;
        if (space > 0) {
            if (err_norm < best) {
                best = err_norm;
                since_best = 0;
            } else if (++since_best >= 12) {
                slot_age.clear();                           // DIIS restart (aimd/qc/scf.py:893-899)
                best = err_norm;
                since_best = 0;
            }
            int slot;
            if ((int)slot_age.size() < space) {
                slot = 0;
                while (std::find(slot_age.begin(), slot_age.end(), slot) != slot_age.end()) ++slot;
            } else {
                slot = slot_age.front();
                slot_age.erase(slot_age.begin());
            }
            slot_age.push_back(slot);
            SCF_CUDA(cudaMemcpyAsync(w.hist_f + (size_t)slot * ne, w.Fo, sizeof(double) * ne,
                                     cudaMemcpyDeviceToDevice, st));
            SCF_CUDA(cudaMemcpyAsync(w.hist_e + (size_t)slot * ne, w.err, sizeof(double) * ne,
                                     cudaMemcpyDeviceToDevice, st));
            // Gram row of the new vector against every stored one (device dots)
            SCF_LIB(cublasSetPointerMode(w.blas, CUBLAS_POINTER_MODE_DEVICE), "pointer mode");
            for (int o : slot_age)
                SCF_LIB(cublasDdot(w.blas, (int)ne, w.hist_e + (size_t)slot * ne, 1, w.hist_e + (size_t)o * ne, 1,
                                   w.red + 4 + o), "cublasDdot");
            SCF_LIB(cublasSetPointerMode(w.blas, CUBLAS_POINTER_MODE_HOST), "pointer mode");
            std::vector<double> row(space);
            SCF_CUDA(cudaMemcpyAsync(row.data(), w.red + 4, sizeof(double) * space, cudaMemcpyDeviceToHost, st));
            SCF_CUDA(cudaStreamSynchronize(st));
            for (int o : slot_age) gram[(size_t)slot * space + o] = gram[(size_t)o * space + slot] = row[o];
            // solve; drop the oldest vectors while the system is singular or the
            // coefficients exceed max_coefficient (aimd/qc/scf.py:551-568)
            while (slot_age.size() > 1) {
                const int k = (int)slot_age.size();
                std::vector<double> B((size_t)k * k);
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j) B[i * k + j] = gram[(size_t)slot_age[i] * space + slot_age[j]];
                double cmax = 0.0;
                const bool ok = pulay(k, B.data(), c.data());
                for (int i = 0; ok && i < k; ++i) cmax = fmax(cmax, std::fabs(c[i]));
                if (ok && cmax <= opt->max_coefficient) break;
                slot_age.erase(slot_age.begin());
            }
            const int k = (int)slot_age.size();
            if (k == 1) c[0] = 1.0;
            std::vector<const double*> hp(k);
            for (int i = 0; i < k; ++i) hp[i] = w.hist_f + (size_t)slot_age[i] * ne;
            SCF_CUDA(cudaMemcpyAsync(w.ptrs, hp.data(), sizeof(double*) * k, cudaMemcpyHostToDevice, st));
            SCF_CUDA(cudaMemcpyAsync(w.coef, c.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
            combine_kernel<<<blocks(ne), 256, 0, st>>>(ne, k, w.ptrs, w.coef, w.Fo);
            SCF_CUDA(cudaGetLastError());
        }
        for (int sp = 0; sp < nspin; ++sp)
            if (int r = aufbau(w, w.Fo + (size_t)sp * m * m, nocc[sp], D + sp * nn, st)) return r;
        e_prev = e_el;
    }
    SCF_CUDA(cudaStreamSynchronize(st));
    *iterations = it > opt->max_iter ? opt->max_iter : it;
    *status = conv ? AIMD_SCF_CONVERGED : AIMD_SCF_MAX_ITER;
    return AIMD_OK;
}

extern "C" int aimd_scf_release(aimd_ctx* ctx) {
    // frees the driver's workspace of this context (call before aimd_destroy)
    Work* w = work_for(ctx, -1, -1, -1);
    release(*w);
    return AIMD_OK;
}
