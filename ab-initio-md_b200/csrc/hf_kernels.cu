// B200 (sm_100a) Hartree-Fock integral engine: C-ABI entry points.
//
// A context owns the device copy of one basis (contraction blocks for the
// two-electron kernels, segmented shells for the one-electron kernels) and
// every geometry-dependent buffer (primitive-pair records, Schwarz bounds,
// the class-sorted pair order and the quartet prefix scans). All device
// memory is allocated in aimd_create; the per-step calls allocate nothing
// and run on the caller's stream.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/aimd_b200.h"
#include "hf_launch.h"

using namespace hf;

namespace {

#define CK(call)                                                     \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) {                                     \
            snprintf(g_err, sizeof g_err, "%s: %s", #call, cudaGetErrorString(e_)); \
            return AIMD_ERR_CUDA;                                    \
        }                                                            \
    } while (0)

thread_local char g_err[512] = "";

template <typename T>
cudaError_t dalloc(T** p, size_t n) { return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)); }

}  // namespace

struct aimd_ctx {
    int natm, nao, nblock, nshell, npair, nspair;
    int nsm;
    // blocks
    int *blk_atom, *blk_l, *blk_ncon, *blk_ao, *blk_p0, *blk_np;
    double *blk_exp, *blk_coef;
    // shells (one-electron)
    int *sh_atom, *sh_l, *sh_ao, *sh_p0, *sh_np, *sp_i, *sp_j;
    double *sh_exp, *sh_coef, *charges;
    int sp_cls_start[7];
    // pairs
    int *pa, *pb, *npp;
    int64_t* slot;
    double* rec;
    int64_t nrec;
    double* Q;
    int cls_start[NCLS + 1];
    int* by_class;          // pair indices grouped by class (static)
    int* idx_in;            // 0..npair-1
    int* tmp_idx;           // pair order after the Q sort
    int* seg_id;            // segment of each pair (geometry dependent)
    int* seg_keys;          // segment of each Q-sorted position
    int* seg_keys_out;
    int* seg_start;         // [NSEG + 1] (device)
    double* tmpQ;
    double* sortedQ;
    int* sorted;
    int64_t* counts_jk;     // [NSEG][npair + 1] kept ket prefix per (ket segment, bra position)
    int64_t* counts_g;
    int64_t* counts_d;      // difference-density builds (threshold changes every call)
    double* bmax;           // [nblock][nblock] max |D| per block pair
    double* dmax;           // [1] max over bmax
    double* jkfix;          // [1] fixed-point scale of the J/K accumulators
    int* plan;              // work plans of the class kernels (LaunchEnv::plan_of)
    int* plan_next;         // their chunk counters
    // launch shape (aimd_set_launch_shape): work-plan chunks per resident
    // CTA, primitive quartets per split column item
    int plan_chunks = 8;
    int item_pq = ITEM_PQ;
    double* bmc;            // gradient: [nblock][nblock] max |Dc| and max over x of |Dx|
    double* bmx;
    cudaStream_t cls_stream[NCLS];
    cudaEvent_t ev_fork, ev_join[NCLS];
    int maxbp[NCLS];        // largest primitive-pair count of a block pair, per class
    double thr_jk = -1.0, thr_g = -1.0;
    // mixed precision: quartets with Q1 Q2 < fp32_cutoff run in FP32
    // (0: all FP64); counts_hi is the FP64 prefix table, built at thr_hi
    double fp32_cutoff = 0.0, thr_hi = -1.0;
    int64_t* counts_hi;
    int64_t* counts_hi_d;   // difference builds: FP64 prefix at fp32_cutoff / max|dD| (per call)
    void* cub_tmp;
    size_t cub_bytes;
    double* pos;            // [natm][3] device copy of the current geometry
    // fixed-point accumulators (order-independent sums): J and K of one
    // density, the nuclear gradient
    facc *jacc = nullptr, *kacc = nullptr, *gacc = nullptr;
    std::vector<double> charges_host;   // nuclear charges (host copy)
    // J/K: bra K rows in global memory for every class (otherwise only where
    // the shared rows would not fit); AIMD_JK_GLOBAL_K_ROWS=1 at creation
    int jk_global_rows = 0;
    bool have_geometry = false;
    uint64_t launches = 0;
};

extern "C" const char* aimd_last_error(void) { return g_err; }

extern "C" int aimd_create(aimd_ctx** out, int natm, int nao, int nblock, const int* blk_atom, const int* blk_l,
                           const int* blk_ncon, const int* blk_ao, const int* blk_p0, const int* blk_np, int nbprim,
                           const double* blk_exp, const double* blk_coef, int nshell, const int* sh_atom,
                           const int* sh_l, const int* sh_ao, const int* sh_p0, const int* sh_np, int nsprim,
                           const double* sh_exp, const double* sh_coef, const double* charges) {
    if (!out || natm <= 0 || nao <= 0 || nblock <= 0 || nshell <= 0) {
        snprintf(g_err, sizeof g_err, "aimd_create: empty basis");
        return AIMD_ERR_ARG;
    }
    for (int b = 0; b < nblock; ++b)
        if (blk_l[b] < 0 || blk_l[b] > LMAX || blk_ncon[b] < 1 || blk_ncon[b] > ncon_cap(blk_l[b])) {
            snprintf(g_err, sizeof g_err, "aimd_create: block %d has l=%d ncon=%d (supported l<=%d, ncon<=cap)", b,
                     blk_l[b], blk_ncon[b], LMAX);
            return AIMD_ERR_UNSUPPORTED;
        }
    for (int s = 0; s < nshell; ++s)
        if (sh_l[s] < 0 || sh_l[s] > LMAX) {
            snprintf(g_err, sizeof g_err, "aimd_create: shell %d has l=%d > %d", s, sh_l[s], LMAX);
            return AIMD_ERR_UNSUPPORTED;
        }
    auto* c = new aimd_ctx();
    {
        const char* kg = getenv("AIMD_JK_GLOBAL_K_ROWS");
        c->jk_global_rows = kg && kg[0] == '1' ? 1 : 0;
    }
    c->natm = natm;
    c->nao = nao;
    c->nblock = nblock;
    c->nshell = nshell;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev));
    auto up_i = [&](int** d, const int* h, size_t n) -> cudaError_t {
        cudaError_t e = dalloc(d, n);
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*d, h, n * sizeof(int), cudaMemcpyHostToDevice);
    };
    auto up_d = [&](double** d, const double* h, size_t n) -> cudaError_t {
        cudaError_t e = dalloc(d, n);
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*d, h, n * sizeof(double), cudaMemcpyHostToDevice);
    };
    CK(up_i(&c->blk_atom, blk_atom, nblock));
    CK(up_i(&c->blk_l, blk_l, nblock));
    CK(up_i(&c->blk_ncon, blk_ncon, nblock));
    CK(up_i(&c->blk_ao, blk_ao, nblock));
    CK(up_i(&c->blk_p0, blk_p0, nblock));
    CK(up_i(&c->blk_np, blk_np, nblock));
    CK(up_d(&c->blk_exp, blk_exp, nbprim));
    CK(up_d(&c->blk_coef, blk_coef, 2 * (size_t)nbprim));
    CK(up_i(&c->sh_atom, sh_atom, nshell));
    CK(up_i(&c->sh_l, sh_l, nshell));
    CK(up_i(&c->sh_ao, sh_ao, nshell));
    CK(up_i(&c->sh_p0, sh_p0, nshell));
    CK(up_i(&c->sh_np, sh_np, nshell));
    CK(up_d(&c->sh_exp, sh_exp, nsprim));
    CK(up_d(&c->sh_coef, sh_coef, nsprim));
    CK(up_d(&c->charges, charges, natm));
    c->charges_host.assign(charges, charges + natm);
    CK(dalloc(&c->pos, 3 * (size_t)natm));
    CK(dalloc(&c->jacc, (size_t)nao * nao));
    CK(dalloc(&c->kacc, (size_t)nao * nao));
    CK(dalloc(&c->gacc, 3 * (size_t)natm));
    // shell pairs (si >= sj) grouped by class (l_i >= l_j after orientation)
    {
        std::vector<int> pi, pj;
        int k = 0;
        for (int cl = 0; cl < NCLS; ++cl) {
            c->sp_cls_start[cl] = k;
            for (int i = 0; i < nshell; ++i)
                for (int j = 0; j <= i; ++j) {
                    int a = i, b = j;
                    if (sh_l[a] < sh_l[b]) std::swap(a, b);
                    if (pcls(sh_l[a], sh_l[b]) != cl) continue;
                    pi.push_back(a);
                    pj.push_back(b);
                    ++k;
                }
        }
        c->sp_cls_start[NCLS] = k;
        c->nspair = k;
        CK(up_i(&c->sp_i, pi.data(), pi.size()));
        CK(up_i(&c->sp_j, pj.data(), pj.size()));
    }
    // block pairs: orientation, class, record slots
    {
        const int np = nblock * (nblock + 1) / 2;
        c->npair = np;
        std::vector<int> pa(np), pb(np), cls(np);
        std::vector<int64_t> slot(np);
        int64_t nrec = 0;
        int ip = 0;
        for (int i = 0; i < nblock; ++i)
            for (int j = 0; j <= i; ++j, ++ip) {
                int a = i, b = j;
                if (blk_l[a] < blk_l[b]) std::swap(a, b);
                pa[ip] = a;
                pb[ip] = b;
                cls[ip] = pcls(blk_l[a], blk_l[b]);
                slot[ip] = nrec;
                nrec += (int64_t)blk_np[a] * blk_np[b];
            }
        c->nrec = nrec;
        std::vector<int> by;
        by.reserve(np);
        for (int cl = 0; cl < NCLS; ++cl) {
            c->cls_start[cl] = (int)by.size();
            for (int p = 0; p < np; ++p)
                if (cls[p] == cl) by.push_back(p);
        }
        c->cls_start[NCLS] = np;
        std::vector<int> iota(np);
        for (int p = 0; p < np; ++p) iota[p] = p;
        CK(up_i(&c->pa, pa.data(), np));
        CK(up_i(&c->pb, pb.data(), np));
        CK(up_i(&c->by_class, by.data(), np));
        CK(up_i(&c->idx_in, iota.data(), np));
        CK(dalloc(&c->tmp_idx, np));
        CK(dalloc(&c->seg_id, np));
        CK(dalloc(&c->seg_keys, np));
        CK(dalloc(&c->seg_keys_out, np));
        CK(dalloc(&c->seg_start, NSEG + 1));
        CK(dalloc(&c->tmpQ, np));
        CK(dalloc(&c->slot, np));
        CK(cudaMemcpy(c->slot, slot.data(), np * sizeof(int64_t), cudaMemcpyHostToDevice));
        CK(dalloc(&c->npp, np));
        CK(dalloc(&c->rec, (size_t)nrec * PPW));
        CK(dalloc(&c->Q, np));
        CK(dalloc(&c->sortedQ, np));
        CK(dalloc(&c->sorted, np));
        CK(dalloc(&c->counts_jk, (size_t)NSEG * (np + 1)));
        CK(dalloc(&c->counts_g, (size_t)NSEG * (np + 1)));
        CK(dalloc(&c->counts_d, (size_t)NSEG * (np + 1)));
        CK(dalloc(&c->counts_hi_d, (size_t)NSEG * (np + 1)));
        CK(dalloc(&c->counts_hi, (size_t)NSEG * (np + 1)));
        CK(dalloc(&c->bmax, (size_t)nblock * nblock));
        CK(dalloc(&c->dmax, 1));
        CK(dalloc(&c->jkfix, 1));
        CK(dalloc(&c->plan, (size_t)2 * NCLS * (np + NCLS)));
        CK(dalloc(&c->plan_next, (size_t)2 * NCLS * NCLS));
        CK(dalloc(&c->bmc, (size_t)nblock * nblock));
        CK(dalloc(&c->bmx, (size_t)nblock * nblock));
        for (int cl = 0; cl < NCLS; ++cl) c->maxbp[cl] = 1;
        for (int p = 0; p < np; ++p)
            c->maxbp[cls[p]] = std::max(c->maxbp[cls[p]], blk_np[pa[p]] * blk_np[pb[p]]);
        size_t b1 = 0, b2 = 0;
        CK(cub::DeviceRadixSort::SortPairsDescending(nullptr, b1, c->Q, c->tmpQ, c->idx_in, c->tmp_idx, np));
        CK(cub::DeviceRadixSort::SortPairs(nullptr, b2, c->seg_keys, c->seg_keys_out, c->tmp_idx, c->sorted, np));
        c->cub_bytes = std::max(b1, b2);
        CK(cudaMalloc(&c->cub_tmp, c->cub_bytes));
    }
    for (int i = 0; i < NCLS; ++i) {
        CK(cudaStreamCreateWithFlags(&c->cls_stream[i], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    *out = c;
    return AIMD_OK;
}

extern "C" int aimd_destroy(aimd_ctx* c) {
    if (!c) return AIMD_OK;
    void* ptrs[] = {c->blk_atom, c->blk_l, c->blk_ncon, c->blk_ao, c->blk_p0, c->blk_np, c->blk_exp, c->blk_coef,
                    c->sh_atom, c->sh_l, c->sh_ao, c->sh_p0, c->sh_np, c->sp_i, c->sp_j, c->sh_exp, c->sh_coef,
                    c->charges, c->pa, c->pb, c->npp, c->slot, c->rec, c->Q, c->by_class, c->idx_in,
                    c->tmp_idx, c->seg_id, c->seg_keys, c->seg_keys_out, c->seg_start, c->tmpQ, c->sortedQ,
                    c->sorted, c->counts_jk, c->counts_g, c->counts_d, c->bmax, c->dmax, c->jkfix, c->plan, c->plan_next, c->bmc, c->bmx, c->counts_hi, c->counts_hi_d, c->cub_tmp, c->pos, c->jacc, c->kacc, c->gacc};
    for (void* p : ptrs) cudaFree(p);
    for (int i = 0; i < NCLS; ++i) {
        if (c->cls_stream[i]) cudaStreamDestroy(c->cls_stream[i]);
        if (c->ev_join[i]) cudaEventDestroy(c->ev_join[i]);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    delete c;
    return AIMD_OK;
}

// ------------------------------------------------------------ geometry

namespace {

// Primitive pairs of each block pair with mu |A-B|^2 <= 50 (the reference's
// PRIM_CUTOFF, aimd/qc/integrals.py:506-510), compacted into the pair's slot.
__global__ void pair_prep_kernel(int npair, const int* pa, const int* pb, const int64_t* slot, const int* blk_atom,
                                 const int* blk_ncon, const int* blk_p0, const int* blk_np, const double* exps,
                                 const double* coefs, const double* pos, int* npp, double* rec) {
    const int ip = blockIdx.x * blockDim.x + threadIdx.x;
    if (ip >= npair) return;
    const int A = pa[ip], B = pb[ip];
    const int iA = blk_atom[A], iB = blk_atom[B];
    const double ABx = pos[3 * iA] - pos[3 * iB], ABy = pos[3 * iA + 1] - pos[3 * iB + 1],
                 ABz = pos[3 * iA + 2] - pos[3 * iB + 2];
    const double r2 = ABx * ABx + ABy * ABy + ABz * ABz;
    // contraction products in compact order: index ca * nB + cb over the
    // block's actual contractions (ca < nA, cb < nB), zeros after them
    const int nA = blk_ncon[A], nB = blk_ncon[B];
    double* out = rec + slot[ip] * PPW;
    int n = 0;
    for (int ka = blk_p0[A]; ka < blk_p0[A] + blk_np[A]; ++ka) {
        const double a = exps[ka];
        for (int kb = blk_p0[B]; kb < blk_p0[B] + blk_np[B]; ++kb) {
            const double b = exps[kb], p = a + b, mu = a * b / p;
            if (!(mu * r2 <= 50.0)) continue;
            double* r = out + (size_t)n * PPW;
            const double bp = b / p, ap = a / p;
            r[0] = a;
            r[1] = b;
            r[2] = exp(-mu * r2);
            r[3] = pos[3 * iA] - bp * ABx;
            r[4] = pos[3 * iA + 1] - bp * ABy;
            r[5] = pos[3 * iA + 2] - bp * ABz;
            r[6] = -bp * ABx;
            r[7] = -bp * ABy;
            r[8] = -bp * ABz;
            r[9] = ap * ABx;
            r[10] = ap * ABy;
            r[11] = ap * ABz;
            for (int i = 0; i < 4; ++i) r[12 + i] = 0.0;
            for (int ca = 0; ca < nA; ++ca)
                for (int cb = 0; cb < nB; ++cb) r[12 + ca * nB + cb] = coefs[2 * ka + ca] * coefs[2 * kb + cb];
            ++n;
        }
    }
    npp[ip] = n;
}

// Segment of each pair: angular class, primitive-pair bucket, contraction count.
__global__ void segment_kernel(int npair, const int* pa, const int* pb, const int* blk_l, const int* blk_ncon,
                               const int* npp, int* seg_id) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npair) return;
    const int A = pa[p], B = pb[p];
    const int nc = blk_ncon[A] * blk_ncon[B];
    const int cb = nc >= 4 ? 2 : (nc >= 2 ? 1 : 0);
    seg_id[p] = pcls(blk_l[A], blk_l[B]) * NSUB + npp_bucket(npp[p]) * NCONB + cb;
}

__global__ void gather_seg_kernel(int n, const int* order, const int* seg_id, int* keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = seg_id[order[i]];
}

__global__ void gather_q_kernel(int n, const int* order, const double* Q, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = Q[order[i]];
}

// seg_start[y] = first sorted position with segment >= y (keys sorted ascending).
__global__ void seg_start_kernel(int n, const int* keys, int* seg_start) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y > NSEG) return;
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < y) lo = mid + 1; else hi = mid;
    }
    seg_start[y] = lo;
}

struct ClsStart { int v[NCLS + 1]; };

// counts[y][s] = number of ket pairs of segment y (a Q-sorted prefix) kept
// with the bra at sorted position s (angular class X >= class of y),
// Q_s Q_j >= thr; for y in class X only positions j <= s (each unordered
// pair of pairs once).
__global__ void quartet_count_kernel(int npair, ClsStart cs, const int* seg_start, const double* sortedQ, double thr,
                                     const double* thr_div, double thr_floor, int64_t* counts) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    // density-weighted enumeration: max(floor, thr / max|D|)
    if (thr_div) thr = *thr_div > 0.0 ? fmax(thr_floor, thr / *thr_div) : INFINITY;
    if (s > npair) return;
    if (s == npair) {
        for (int y = 0; y < NSEG; ++y) counts[(size_t)y * (npair + 1) + npair] = 0;
        return;
    }
    int X = 0;
    while (s >= cs.v[X + 1]) ++X;
    const double qs = sortedQ[s];
    for (int y = 0; y < NSEG; ++y) {
        int64_t cnt = 0;
        const int cy = y / NSUB;
        if (cy <= X) {
            const int y0 = seg_start[y], y1 = seg_start[y + 1];
            int lo = y0, hi = y1;       // first j with qs*Q_j < thr
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (qs * sortedQ[mid] >= thr) lo = mid + 1; else hi = mid;
            }
            cnt = lo - y0;
            if (cy == X) {
                const int64_t cap = (int64_t)s + 1 - y0;
                cnt = cap <= 0 ? 0 : (cnt > cap ? cap : cnt);
            }
        }
        counts[(size_t)y * (npair + 1) + s] = cnt;
    }
}

// bmax[I][J] = max over the functions of blocks I, J and the sets of |D|
__global__ void block_dmax_kernel(int nblock, int nao, int nset, const int* blk_l, const int* blk_ncon,
                                  const int* blk_ao, const double* D, double* bmax) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nblock * nblock) return;
    const int I = i / nblock, J = i % nblock;
    const int nI = blk_ncon[I] * ncart(blk_l[I]), nJ = blk_ncon[J] * ncart(blk_l[J]);
    const size_t nn = (size_t)nao * nao;
    double m = 0.0;
    for (int s = 0; s < nset; ++s)
        for (int a = 0; a < nI; ++a)
            for (int b = 0; b < nJ; ++b) m = fmax(m, fabs(D[s * nn + (size_t)(blk_ao[I] + a) * nao + blk_ao[J] + b]));
    bmax[i] = m;
}

// out = acc / scale (add = 0) or out += acc / scale (add = 1); the scale is
// *scale_p when that is given (a device scalar), else scale
__global__ void from_fixed_kernel(size_t n, const facc* acc, const double* scale_p, double scale, double* out,
                                  int add) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = from_fixed(acc[i], scale_p ? *scale_p : scale);
    out[i] = add ? out[i] + v : v;
}
void from_fixed(cudaStream_t st, size_t n, const facc* acc, const double* scale_p, double scale, double* out,
                int add) {
    from_fixed_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, acc, scale_p, scale, out, add);
}

// *out = max of x[0 .. n); fix (optional) = jk_fix_for(*out)
__global__ void max_reduce_kernel(int n, const double* x, double* out, double* fix) {
    __shared__ double sm[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, x[i]);
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *out = sm[0];
        if (fix) *fix = jk_fix_for(sm[0]);
    }
}

PairView pair_view(aimd_ctx* c) { return PairView{c->pa, c->pb, c->slot, c->npp, c->rec}; }
BlockView block_view(aimd_ctx* c) { return BlockView{c->blk_atom, c->blk_l, c->blk_ncon, c->blk_ao}; }

QuartetArgs quartet_args(aimd_ctx* c, const int64_t* counts) {
    QuartetArgs q;
    q.pv = pair_view(c);
    q.bv = block_view(c);
    q.sorted = c->sorted;
    q.sortedQ = c->sortedQ;
    q.counts = counts;
    q.counts_hi = nullptr;
    q.seg_start = c->seg_start;
    q.npair = c->npair;
    for (int i = 0; i <= NCLS; ++i) q.cls_start[i] = c->cls_start[i];
    q.nao = c->nao;
    return q;
}

int build_counts(aimd_ctx* c, double thr, int64_t* counts, cudaStream_t st, const double* thr_div = nullptr,
                 double thr_floor = 0.0) {
    ClsStart cs;
    for (int i = 0; i <= NCLS; ++i) cs.v[i] = c->cls_start[i];
    const int n = c->npair + 1;
    quartet_count_kernel<<<(n + 127) / 128, 128, 0, st>>>(c->npair, cs, c->seg_start, c->sortedQ, thr, thr_div,
                                                           thr_floor, counts);
    ++c->launches;
    CK(cudaGetLastError());
    return AIMD_OK;
}

int ncls_pairs(aimd_ctx* c, int cl) { return c->cls_start[cl + 1] - c->cls_start[cl]; }

LaunchEnv launch_env(aimd_ctx* c) {
    LaunchEnv e;
    for (int cl = 0; cl < NCLS; ++cl) {
        e.cls_count[cl] = ncls_pairs(c, cl);
        e.maxbp[cl] = c->maxbp[cl];
    }
    for (int cl = 0; cl <= NCLS; ++cl) e.cls_start[cl] = c->cls_start[cl];
    e.nao = c->nao;
    e.natm = c->natm;
    e.by_class = c->by_class;
    e.Q = c->Q;
    e.nsm = c->nsm;
    e.plan = c->plan;
    e.plan_next = c->plan_next;
    e.plan_stride = c->npair + NCLS;
    return e;
}

// Work plan of the (CX, CY, RT) launch (one CTA of PLAN_THREADS): per bra
// of class CX its chunk count ceil(W / target), target = max(total W /
// parts, PLAN_MIN_WORK) with parts = chunks per resident CTA x resident
// CTAs, as an exclusive prefix in off[0 .. nbra]; the launch's chunk
// counter is zeroed.
constexpr int PLAN_THREADS = 1024;
constexpr int64_t PLAN_MIN_WORK = 4096;

template <typename T>
__device__ T block_sum(T v, T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    T t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;
}

template <int CX, int CY, typename RT>
__device__ void plan_launch(const QuartetArgs& q, int* off, int* next, int parts) {
    __shared__ int64_t red[PLAN_THREADS / 32];
    __shared__ int ired[PLAN_THREADS / 32];
    const int nbra = q.cls_start[CX + 1] - q.cls_start[CX];
    const int per = (nbra + PLAN_THREADS - 1) / PLAN_THREADS;
    const int b0 = min(nbra, (int)threadIdx.x * per), b1 = min(nbra, b0 + per);
    int64_t w = 0;
    for (int b = b0; b < b1; ++b) w += bra_work<CX, CY, RT>(q, q.cls_start[CX] + b);
    const int64_t W = block_sum(w, red);
    int64_t target = W / parts;
    if (target < PLAN_MIN_WORK) target = PLAN_MIN_WORK;
    int cnt = 0;
    for (int b = b0; b < b1; ++b) {
        const int64_t wb = bra_work<CX, CY, RT>(q, q.cls_start[CX] + b);
        off[b] = (int)((wb + target - 1) / target);
        cnt += off[b];
    }
    // exclusive scan of the per-thread counts (threads in index order)
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    if (lane == 31) ired[warp] = incl;
    __syncthreads();
    int base = incl - cnt;
    for (int w2 = 0; w2 < warp; ++w2) base += ired[w2];
    for (int b = b0; b < b1; ++b) {
        const int k = off[b];
        off[b] = base;
        base += k;
    }
    if (threadIdx.x == PLAN_THREADS - 1) {
        off[nbra] = base;                               // the last thread ends at the total
        *next = 0;
    }
}

// one CTA per (bra class, ket class <= bra class, type): blockIdx.x = pair
// index CX (CX + 1) / 2 + CY, blockIdx.y = type (0: FP64 ranges, 1: FP32)
__global__ void __launch_bounds__(PLAN_THREADS) plan_kernel(QuartetArgs q, int* plan, int* plan_next, int stride,
                                                            int parts) {
    int cx = 0;
    while ((cx + 1) * (cx + 2) / 2 <= (int)blockIdx.x) ++cx;
    const int cy = blockIdx.x - cx * (cx + 1) / 2, rt = blockIdx.y;
    int* off = plan + (size_t)(rt * NCLS + cy) * stride + q.cls_start[cx] + cx;
    int* next = plan_next + (rt * NCLS + cx) * NCLS + cy;
#define AIMD_PLAN(X, Y)                                                         \
    if (cx == X && cy == Y) {                                                   \
        if (rt == 0) plan_launch<X, Y, double>(q, off, next, parts);           \
        else plan_launch<X, Y, float>(q, off, next, parts);                    \
    }
    AIMD_PLAN(0, 0)
    AIMD_PLAN(1, 0) AIMD_PLAN(1, 1)
    AIMD_PLAN(2, 0) AIMD_PLAN(2, 1) AIMD_PLAN(2, 2)
    AIMD_PLAN(3, 0) AIMD_PLAN(3, 1) AIMD_PLAN(3, 2) AIMD_PLAN(3, 3)
    AIMD_PLAN(4, 0) AIMD_PLAN(4, 1) AIMD_PLAN(4, 2) AIMD_PLAN(4, 3) AIMD_PLAN(4, 4)
    AIMD_PLAN(5, 0) AIMD_PLAN(5, 1) AIMD_PLAN(5, 2) AIMD_PLAN(5, 3) AIMD_PLAN(5, 4) AIMD_PLAN(5, 5)
#undef AIMD_PLAN
}

// Plans of every class launch of one call (mixed: the FP32 ones too), on st
// before the class streams fork.
void plan_launches(aimd_ctx* c, const QuartetArgs& q, bool mixed, cudaStream_t st) {
    plan_kernel<<<dim3(NCLS * (NCLS + 1) / 2, mixed ? 2 : 1), PLAN_THREADS, 0, st>>>(q, c->plan, c->plan_next,
                                                                                   c->npair + NCLS,
                                                                                   c->plan_chunks * 2 * c->nsm);
    ++c->launches;
}

// all (CX, CY <= CX) gradient kernels of bra class CX, in order on one stream
template <int CX>
cudaError_t launch_grad_class(const LaunchEnv& e, const GradArgs& a, cudaStream_t st) {
    cudaError_t r = cudaSuccess;
    const bool mixed = a.q.counts_hi != nullptr;
#define AIMD_G1(X, Y)                                                             \
    if (r == cudaSuccess && CX == X) r = launch_grad_c##X##_##Y(e, a, st);       \
    if (r == cudaSuccess && CX == X && mixed) r = launch_grad32_c##X##_##Y(e, a, st);
    AIMD_G1(0, 0)
    AIMD_G1(1, 0) AIMD_G1(1, 1)
    AIMD_G1(2, 0) AIMD_G1(2, 1) AIMD_G1(2, 2)
    AIMD_G1(3, 0) AIMD_G1(3, 1) AIMD_G1(3, 2) AIMD_G1(3, 3)
    AIMD_G1(4, 0) AIMD_G1(4, 1) AIMD_G1(4, 2) AIMD_G1(4, 3) AIMD_G1(4, 4)
    AIMD_G1(5, 0) AIMD_G1(5, 1) AIMD_G1(5, 2) AIMD_G1(5, 3) AIMD_G1(5, 4) AIMD_G1(5, 5)
#undef AIMD_G1
    return r;
}

// kernel launches of one class step: J/K one per type, the gradient one
// per (bra class, non-empty ket class) and type
int cls_size(aimd_ctx* c, int cl) { return c->cls_start[cl + 1] - c->cls_start[cl]; }
int jk_launches(aimd_ctx* c, int cl, bool mixed) {
    if (cls_size(c, cl) == 0) return 0;
    int n = 1;
    if (cl >= 1) {          // split bra classes: one kernel per non-empty ket class
        n = 0;
        for (int y = 0; y <= cl; ++y) n += cls_size(c, y) > 0 ? 1 : 0;
    }
    return mixed ? 2 * n : n;
}
int grad_launches(aimd_ctx* c, int cl, bool mixed) {
    int n = 0;
    for (int y = 0; y <= cl; ++y) n += (cls_size(c, cl) > 0 && cls_size(c, y) > 0) ? 1 : 0;
    return mixed ? 2 * n : n;
}

inline cudaError_t first_error(cudaError_t a, cudaError_t b) { return a != cudaSuccess ? a : b; }

int class_status(aimd_ctx* c, cudaError_t r, const char* what, int cl, int nlaunch) {
    if (r == cudaSuccess) {
        c->launches += nlaunch;
        return AIMD_OK;
    }
    if (r == cudaErrorInvalidConfiguration) {
        snprintf(g_err, sizeof g_err, "%s (pair class %d): shared memory beyond the 227 KB per-CTA limit",
                 what, cl);
        return AIMD_ERR_UNSUPPORTED;
    }
    snprintf(g_err, sizeof g_err, "%s (pair class %d): %s", what, cl, cudaGetErrorString(r));
    return AIMD_ERR_CUDA;
}

#define AIMD_EACH_CLASS(CALL, WHAT)                                         \
    do {                                                                    \
        int r_;                                                             \
        if ((r_ = class_status(c, CALL(0), WHAT, 0, cls_size(c, 0) > 0))) return r_;  \
        if ((r_ = class_status(c, CALL(1), WHAT, 1, cls_size(c, 1) > 0))) return r_;  \
        if ((r_ = class_status(c, CALL(2), WHAT, 2, cls_size(c, 2) > 0))) return r_;  \
        if ((r_ = class_status(c, CALL(3), WHAT, 3, cls_size(c, 3) > 0))) return r_;  \
        if ((r_ = class_status(c, CALL(4), WHAT, 4, cls_size(c, 4) > 0))) return r_;  \
        if ((r_ = class_status(c, CALL(5), WHAT, 5, cls_size(c, 5) > 0))) return r_;  \
    } while (0)

// The six class launches of one call run concurrently on the context's
// class streams, forked from and joined back into the caller's stream, so
// the long-running d-shell classes overlap the others.
#define AIMD_EACH_CLASS_CONCURRENT(CALL, WHAT, NLAUNCH)                               \
    do {                                                                              \
        CK(cudaEventRecord(c->ev_fork, st));                                          \
        int r_ = AIMD_OK;                                                             \
        for (int x_ = NCLS - 1; x_ >= 0 && r_ == AIMD_OK; --x_) {                     \
            CK(cudaStreamWaitEvent(c->cls_stream[x_], c->ev_fork, 0));                \
            cudaStream_t cs_ = c->cls_stream[x_];                                     \
            cudaError_t e_ = cudaSuccess;                                             \
            switch (x_) {                                                             \
                case 0: e_ = CALL(0, cs_); break;                                     \
                case 1: e_ = CALL(1, cs_); break;                                     \
                case 2: e_ = CALL(2, cs_); break;                                     \
                case 3: e_ = CALL(3, cs_); break;                                     \
                case 4: e_ = CALL(4, cs_); break;                                     \
                default: e_ = CALL(5, cs_); break;                                    \
            }                                                                         \
            r_ = class_status(c, e_, WHAT, x_, NLAUNCH(x_));                          \
            CK(cudaEventRecord(c->ev_join[x_], cs_));                                 \
            CK(cudaStreamWaitEvent(st, c->ev_join[x_], 0));                           \
        }                                                                             \
        if (r_) return r_;                                                            \
    } while (0)

// The FP64-prefix table of the mixed-precision path (nullptr when off).
int hi_counts(aimd_ctx* c, cudaStream_t st, const int64_t** out) {
    *out = nullptr;
    if (!(c->fp32_cutoff > 0.0)) return AIMD_OK;
    if (c->thr_hi != c->fp32_cutoff) {
        if (int r = build_counts(c, c->fp32_cutoff, c->counts_hi, st)) return r;
        c->thr_hi = c->fp32_cutoff;
    }
    *out = c->counts_hi;
    return AIMD_OK;
}

}  // namespace

extern "C" int aimd_set_fp32_cutoff(aimd_ctx* c, double cutoff) {
    if (!c || !(cutoff >= 0.0) || !std::isfinite(cutoff)) {
        snprintf(g_err, sizeof g_err, "aimd_set_fp32_cutoff: cutoff must be finite and >= 0");
        return AIMD_ERR_ARG;
    }
    c->fp32_cutoff = cutoff;
    return AIMD_OK;
}

extern "C" int aimd_set_launch_shape(aimd_ctx* c, int chunks_per_cta, int item_pq) {
    if (!c || chunks_per_cta < 1 || chunks_per_cta > 64 || item_pq < 4 || item_pq > 4096) {
        snprintf(g_err, sizeof g_err,
                 "aimd_set_launch_shape: chunks_per_cta must be in 1..64 and item_pq in 4..4096");
        return AIMD_ERR_ARG;
    }
    c->plan_chunks = chunks_per_cta;
    c->item_pq = item_pq;
    return AIMD_OK;
}

extern "C" int aimd_get_launch_shape(aimd_ctx* c, int* chunks_per_cta, int* item_pq) {
    if (!c || !chunks_per_cta || !item_pq) return AIMD_ERR_ARG;
    *chunks_per_cta = c->plan_chunks;
    *item_pq = c->item_pq;
    return AIMD_OK;
}

extern "C" int aimd_set_geometry(aimd_ctx* c, const double* pos, void* stream) {
    if (!c || !pos) return AIMD_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemcpyAsync(c->pos, pos, 3 * sizeof(double) * c->natm, cudaMemcpyDefault, st));
    const int np = c->npair;
    pair_prep_kernel<<<(np + 127) / 128, 128, 0, st>>>(np, c->pa, c->pb, c->slot, c->blk_atom, c->blk_ncon, c->blk_p0,
                                                        c->blk_np, c->blk_exp, c->blk_coef, c->pos, c->npp, c->rec);
    ++c->launches;
    CK(cudaGetLastError());
    {
        const LaunchEnv e = launch_env(c);
        const QuartetArgs q = quartet_args(c, c->counts_jk);
#define AIMD_SCHWARZ(X) launch_schwarz_c##X(e, q, st)
        AIMD_EACH_CLASS(AIMD_SCHWARZ, "aimd_set_geometry/schwarz");
#undef AIMD_SCHWARZ
    }
    // order: Q descending, then (stable) by segment; segment starts on the device
    const int nbk = (np + 127) / 128;
    segment_kernel<<<nbk, 128, 0, st>>>(np, c->pa, c->pb, c->blk_l, c->blk_ncon, c->npp, c->seg_id);
    size_t bytes = c->cub_bytes;
    CK(cub::DeviceRadixSort::SortPairsDescending(c->cub_tmp, bytes, c->Q, c->tmpQ, c->idx_in, c->tmp_idx, np, 0,
                                                 sizeof(double) * 8, st));
    gather_seg_kernel<<<nbk, 128, 0, st>>>(np, c->tmp_idx, c->seg_id, c->seg_keys);
    bytes = c->cub_bytes;
    CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp, bytes, c->seg_keys, c->seg_keys_out, c->tmp_idx, c->sorted, np, 0,
                                       sizeof(int) * 8, st));
    gather_q_kernel<<<nbk, 128, 0, st>>>(np, c->sorted, c->Q, c->sortedQ);
    seg_start_kernel<<<1, NSEG + 1, 0, st>>>(np, c->seg_keys_out, c->seg_start);
    c->launches += 6;
    CK(cudaGetLastError());
    c->thr_jk = c->thr_g = c->thr_hi = -1.0;
    c->have_geometry = true;
    return AIMD_OK;
}

extern "C" int aimd_schwarz(aimd_ctx* c, double* Q, void* stream) {
    if (!c || !Q || !c->have_geometry) return AIMD_ERR_ARG;
    CK(cudaMemcpyAsync(Q, c->Q, sizeof(double) * c->npair, cudaMemcpyDefault, static_cast<cudaStream_t>(stream)));
    return AIMD_OK;
}

extern "C" int aimd_pair_count(aimd_ctx* c) { return c ? c->npair : 0; }

extern "C" int aimd_jk(aimd_ctx* c, int nset, const double* D, double* J, double* K, double thr, void* stream) {
    if (!c || !D || !J || !K || nset < 1 || !c->have_geometry) return AIMD_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (thr != c->thr_jk) {
        if (int r = build_counts(c, thr, c->counts_jk, st)) return r;
        c->thr_jk = thr;
    }
    const int64_t* hi = nullptr;
    if (int r = hi_counts(c, st, &hi)) return r;
    const bool mixed = hi != nullptr;
    const size_t nn = (size_t)c->nao * c->nao;
    // fixed-point scale of the accumulators from max |D| over the sets
    const int nb2 = c->nblock * c->nblock;
    block_dmax_kernel<<<(nb2 + 127) / 128, 128, 0, st>>>(c->nblock, c->nao, nset, c->blk_l, c->blk_ncon, c->blk_ao, D,
                                                         c->bmax);
    max_reduce_kernel<<<1, 256, 0, st>>>(nb2, c->bmax, c->dmax, c->jkfix);
    c->launches += 2;

    // one pass per density (UHF: alpha and beta)
    const LaunchEnv e = launch_env(c);
    for (int s0 = 0; s0 < nset; ++s0) {
        JKArgs a;
        a.q = quartet_args(c, c->counts_jk);
        a.q.counts_hi = hi;
        a.D = D + s0 * nn;
        a.J = c->jacc;
        a.K = c->kacc;
        a.fix = c->jkfix;
        CK(cudaMemsetAsync(c->jacc, 0, sizeof(facc) * nn, st));
        CK(cudaMemsetAsync(c->kacc, 0, sizeof(facc) * nn, st));
        a.bmax = nullptr;
        a.nblock = c->nblock;
        a.dthr = 0.0;
        a.rbuf = 0;
        a.kglobal = c->jk_global_rows;
        a.item_pq = c->item_pq;
        plan_launches(c, a.q, mixed, st);
#define AIMD_JK(X, S) first_error(launch_jk_c##X(e, a, S), mixed ? launch_jk32_c##X(e, a, S) : cudaSuccess)
#define AIMD_NL(X) jk_launches(c, X, mixed)
        AIMD_EACH_CLASS_CONCURRENT(AIMD_JK, "aimd_jk", AIMD_NL);
#undef AIMD_NL
#undef AIMD_JK
        from_fixed(st, nn, c->jacc, c->jkfix, 0.0, J + s0 * nn, 0);
        from_fixed(st, nn, c->kacc, c->jkfix, 0.0, K + s0 * nn, 0);
        c->launches += 2;
        CK(cudaGetLastError());
    }
    return AIMD_OK;
}

namespace {
// unit symmetric density D_ls = D_sl = 1/2 (l != s), D_ll = 1
__global__ void unit_density_kernel(int n, int l, int s, double* D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n) return;
    const int r = i / n, c = i % n;
    D[i] = ((r == l && c == s) || (r == s && c == l)) ? (l == s ? 1.0 : 0.5) : 0.0;
}
// eri[m][n][l][s] = eri[m][n][s][l] = J[m][n] + J[n][m]
__global__ void scatter_slice_kernel(int n, int l, int s, const double* J, double* eri) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n) return;
    const size_t m = i / n, nn_ = i % n, N = n;
    const double v = J[m * N + nn_] + J[nn_ * N + m];
    eri[((m * N + nn_) * N + l) * N + s] = v;
    eri[((m * N + nn_) * N + s) * N + l] = v;
}
}  // namespace

// J/K accumulators of a change of density (incremental Fock builds): a
// quartet is skipped when Q_ab Q_cd max|dD| < dthr, max over the six block
// pairs of dD that it touches (density-weighted Schwarz screening).
extern "C" int aimd_jk_delta(aimd_ctx* c, int nset, const double* D, double* J, double* K, double thr, double dthr,
                             void* stream) {
    if (!c || !D || !J || !K || nset < 1 || !c->have_geometry || !(dthr > 0.0)) return AIMD_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nn = (size_t)c->nao * c->nao;
    const int nb2 = c->nblock * c->nblock;
    block_dmax_kernel<<<(nb2 + 127) / 128, 128, 0, st>>>(c->nblock, c->nao, nset, c->blk_l, c->blk_ncon, c->blk_ao, D,
                                                         c->bmax);
    max_reduce_kernel<<<1, 256, 0, st>>>(nb2, c->bmax, c->dmax, c->jkfix);
    c->launches += 2;
    CK(cudaGetLastError());
    // enumerate at max(thr, dthr / max|D|): the integral screen still holds,
    // and no quartet that the density-weighted test keeps is missed
    if (int r = build_counts(c, dthr, c->counts_d, st, c->dmax, thr)) return r;
    // mixed precision: a quartet of a difference build contributes at most
    // Q1 Q2 max|dD|, so the FP32 rule is applied to that product, i.e. the
    // FP64 prefix is cut at fp32_cutoff / max|dD|
    const int64_t* hi = nullptr;
    if (c->fp32_cutoff > 0.0) {
        if (int r = build_counts(c, c->fp32_cutoff, c->counts_hi_d, st, c->dmax, 0.0)) return r;
        hi = c->counts_hi_d;
    }
    const bool mixed = hi != nullptr;

    const LaunchEnv e = launch_env(c);
    for (int s0 = 0; s0 < nset; ++s0) {
        JKArgs a;
        a.q = quartet_args(c, c->counts_d);
        a.q.counts_hi = hi;
        a.D = D + s0 * nn;
        a.J = c->jacc;
        a.K = c->kacc;
        a.fix = c->jkfix;
        CK(cudaMemsetAsync(c->jacc, 0, sizeof(facc) * nn, st));
        CK(cudaMemsetAsync(c->kacc, 0, sizeof(facc) * nn, st));
        a.bmax = c->bmax;
        a.nblock = c->nblock;
        a.dthr = dthr;
        a.rbuf = 0;
        a.kglobal = c->jk_global_rows;
        a.item_pq = c->item_pq;
        plan_launches(c, a.q, mixed, st);
#define AIMD_JK(X, S) first_error(launch_jk_c##X(e, a, S), mixed ? launch_jk32_c##X(e, a, S) : cudaSuccess)
#define AIMD_NL(X) jk_launches(c, X, mixed)
        AIMD_EACH_CLASS_CONCURRENT(AIMD_JK, "aimd_jk_delta", AIMD_NL);
#undef AIMD_NL
#undef AIMD_JK
        from_fixed(st, nn, c->jacc, c->jkfix, 0.0, J + s0 * nn, 0);
        from_fixed(st, nn, c->kacc, c->jkfix, 0.0, K + s0 * nn, 0);
        c->launches += 2;
        CK(cudaGetLastError());
    }
    return AIMD_OK;
}

namespace {
// The tensor probes evaluate every quartet in FP64 whatever FP32 cutoff the
// context carries: the cutoff is set aside for the probe and put back after.
struct Fp64Probe {
    aimd_ctx* c;
    double saved;
    explicit Fp64Probe(aimd_ctx* ctx) : c(ctx), saved(ctx->fp32_cutoff) { c->fp32_cutoff = 0.0; }
    ~Fp64Probe() { c->fp32_cutoff = saved; }
};
}  // namespace

// Test and debug sizes only: the tensor is probed column by column through
// the integral-direct Coulomb build (J[D] with D the symmetric unit matrix
// of (l, s) gives (mn|ls)); scratch for D/J/K is allocated here.
extern "C" int aimd_eri_tensor(aimd_ctx* c, double* eri, double thr, void* stream) {
    if (!c || !eri || !c->have_geometry) return AIMD_ERR_ARG;
    const Fp64Probe fp64(c);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = c->nao;
    const size_t nn = (size_t)n * n;
    double* scratch = nullptr;
    CK(cudaMalloc(&scratch, 3 * nn * sizeof(double)));
    double *D = scratch, *J = scratch + nn, *K = scratch + 2 * nn;
    int status = AIMD_OK;
    const int blocks = (int)((nn + 255) / 256);
    for (int l = 0; l < n && status == AIMD_OK; ++l)
        for (int s = 0; s <= l && status == AIMD_OK; ++s) {
            unit_density_kernel<<<blocks, 256, 0, st>>>(n, l, s, D);
            ++c->launches;
            status = aimd_jk(c, 1, D, J, K, thr, stream);
            if (status == AIMD_OK) {
                scatter_slice_kernel<<<blocks, 256, 0, st>>>(n, l, s, J, eri);
                ++c->launches;
            }
        }
    cudaError_t e1 = cudaStreamSynchronize(st);
    cudaFree(scratch);
    if (status != AIMD_OK) return status;
    CK(e1);
    return AIMD_OK;
}

// Scratch of aimd_eri_tensor_static: D, J and K of one probe for up to
// AIMD_ERI_STATIC_MAX_NAO AOs (3 x 128^2 doubles = 384 KiB per device),
// in the module's static device memory instead of cudaMalloc.
static __device__ __align__(256) double g_eri_static_scratch[3 * AIMD_ERI_STATIC_MAX_NAO * AIMD_ERI_STATIC_MAX_NAO];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_eri_static_mu;
double* g_eri_static_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (the first call on each device does this set-up).
int eri_static_scratch(double** out) {
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        snprintf(g_err, sizeof g_err, "aimd_eri_tensor_static: device ordinal %d beyond %d", dev, kMaxDevices);
        return AIMD_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_eri_static_mu);
    if (!g_eri_static_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_eri_static_scratch);
        if (e != cudaSuccess || !p) {
            snprintf(g_err, sizeof g_err, "aimd_eri_tensor_static: cudaGetSymbolAddress: %s",
                     cudaGetErrorString(e));
            return AIMD_ERR_CUDA;
        }
        g_eri_static_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_eri_static_ptr[dev];
    return AIMD_OK;
}
}  // namespace

// aimd_eri_tensor without any allocation: the D/J/K probe scratch is the
// static array above, so nao <= AIMD_ERI_STATIC_MAX_NAO. Nothing in the
// scratch has to start at zero (each probe writes all of D, and aimd_jk
// clears J and K); every element of eri is written. Asynchronous on stream.
extern "C" int aimd_eri_tensor_static(aimd_ctx* c, double* eri, double thr, void* stream) {
    if (!c || !eri || !c->have_geometry) return AIMD_ERR_ARG;
    const int n = c->nao;
    if (n > AIMD_ERI_STATIC_MAX_NAO) {
        snprintf(g_err, sizeof g_err, "aimd_eri_tensor_static: %d AOs exceed the static scratch limit of %d AOs "
                 "(use aimd_eri_tensor)", n, AIMD_ERI_STATIC_MAX_NAO);
        return AIMD_ERR_ARG;
    }
    // the context's buffers must live on the current device, like the scratch
    cudaPointerAttributes pa;
    CK(cudaPointerGetAttributes(&pa, c->rec));
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (pa.device != dev) {
        snprintf(g_err, sizeof g_err, "aimd_eri_tensor_static: context on device %d, current device %d",
                 pa.device, dev);
        return AIMD_ERR_ARG;
    }
    double* scratch = nullptr;
    if (int r = eri_static_scratch(&scratch)) return r;
    const Fp64Probe fp64(c);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nn = (size_t)n * n;
    double *D = scratch, *J = scratch + nn, *K = scratch + 2 * nn;
    const int blocks = (int)((nn + 255) / 256);
    for (int l = 0; l < n; ++l)
        for (int s = 0; s <= l; ++s) {
            unit_density_kernel<<<blocks, 256, 0, st>>>(n, l, s, D);
            ++c->launches;
            if (int r = aimd_jk(c, 1, D, J, K, thr, stream)) return r;
            scatter_slice_kernel<<<blocks, 256, 0, st>>>(n, l, s, J, eri);
            ++c->launches;
        }
    CK(cudaGetLastError());
    return AIMD_OK;
}

extern "C" int aimd_grad2e(aimd_ctx* c, const double* Dc, int nx, const double* Dx, double kfac, double thr,
                           double gamma_bound, double* grad, void* stream) {
    if (!c || !Dc || (nx > 0 && !Dx) || !grad || !c->have_geometry || !(gamma_bound > 0.0)) return AIMD_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // enumerate every quartet that can pass Q1 Q2 max|Gamma| >= thr
    const double thr_enum = thr / gamma_bound;
    if (thr_enum != c->thr_g) {
        if (int r = build_counts(c, thr_enum, c->counts_g, st)) return r;
        c->thr_g = thr_enum;
    }
    CK(cudaMemsetAsync(c->gacc, 0, sizeof(facc) * 3 * c->natm, st));
    const int nb2 = c->nblock * c->nblock;
    block_dmax_kernel<<<(nb2 + 127) / 128, 128, 0, st>>>(c->nblock, c->nao, 1, c->blk_l, c->blk_ncon, c->blk_ao, Dc,
                                                         c->bmc);
    ++c->launches;
    if (nx > 0) {
        block_dmax_kernel<<<(nb2 + 127) / 128, 128, 0, st>>>(c->nblock, c->nao, nx, c->blk_l, c->blk_ncon, c->blk_ao,
                                                             Dx, c->bmx);
        ++c->launches;
    }
    CK(cudaGetLastError());
    const int64_t* hi = nullptr;
    if (int r = hi_counts(c, st, &hi)) return r;
    const bool mixed = hi != nullptr;
    GradArgs a;
    a.q = quartet_args(c, c->counts_g);
    a.q.counts_hi = hi;
    a.Dc = Dc;
    a.Dx = Dx;
    a.nx = nx;
    a.kfac = kfac;
    a.thr = thr;
    a.grad = c->gacc;
    a.natm = c->natm;
    a.rbuf = 0;
    a.bmc = c->bmc;
    a.bmx = c->bmx;
    a.nblock = c->nblock;
    a.item_pq = c->item_pq;
    plan_launches(c, a.q, mixed, st);
    const LaunchEnv e = launch_env(c);
#define AIMD_GRAD(X, S) launch_grad_class<X>(e, a, S)
#define AIMD_NL(X) grad_launches(c, X, mixed)
    AIMD_EACH_CLASS_CONCURRENT(AIMD_GRAD, "aimd_grad2e", AIMD_NL);
#undef AIMD_NL
#undef AIMD_GRAD
    from_fixed(st, 3 * (size_t)c->natm, c->gacc, nullptr, FIX_G, grad, 0);
    ++c->launches;
    CK(cudaGetLastError());
    return AIMD_OK;
}

namespace {
ShellView shell_view(aimd_ctx* c) {
    ShellView s;
    s.nshell = c->nshell;
    s.natm = c->natm;
    s.nao = c->nao;
    s.atom = c->sh_atom;
    s.l = c->sh_l;
    s.ao = c->sh_ao;
    s.p0 = c->sh_p0;
    s.np = c->sh_np;
    s.exps = c->sh_exp;
    s.coefs = c->sh_coef;
    s.pos = c->pos;
    s.charges = c->charges;
    s.pair_i = c->sp_i;
    s.pair_j = c->sp_j;
    return s;
}
}  // namespace

extern "C" int aimd_onee(aimd_ctx* c, const double* origin, double* S, double* T, double* M, double* V,
                         void* stream) {
    if (!c || !S || !T || !M || !V || !c->have_geometry) return AIMD_ERR_ARG;
    int n = 0;
    cudaError_t r = launch_onee(launch_env(c), shell_view(c), c->sp_cls_start, origin, S, T, M, V,
                                static_cast<cudaStream_t>(stream), &n);
    c->launches += n;
    CK(r);
    return AIMD_OK;
}

extern "C" int aimd_onee_grad(aimd_ctx* c, const double* W, const double* D, double* grad, void* stream) {
    if (!c || !W || !D || !grad || !c->have_geometry) return AIMD_ERR_ARG;
    int n = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemsetAsync(c->gacc, 0, sizeof(facc) * 3 * c->natm, st));
    cudaError_t r = launch_onee_grad(launch_env(c), shell_view(c), c->sp_cls_start, W, D, c->gacc, st, &n);
    if (r == cudaSuccess) {
        from_fixed(st, 3 * (size_t)c->natm, c->gacc, nullptr, FIX_G, grad, 1);
        ++n;
        r = cudaGetLastError();
    }
    c->launches += n;
    if (r == cudaErrorInvalidConfiguration) {
        snprintf(g_err, sizeof g_err, "aimd_onee_grad: too many atoms for the shared accumulator");
        return AIMD_ERR_UNSUPPORTED;
    }
    CK(r);
    return AIMD_OK;
}

extern "C" int aimd_quartet_counts(aimd_ctx* c, int which, int64_t* out_host) {
    // kept quartets per class pair (bra class X, ket class Y <= X), 6 x 6
    // row-major, for the J/K list (which = 0) or the gradient list (which = 1)
    if (!c || !out_host || !c->have_geometry) return AIMD_ERR_ARG;
    const int64_t* counts = which ? c->counts_g : c->counts_jk;
    const int n = c->npair + 1;
    std::vector<int64_t> h((size_t)NSEG * n);
    CK(cudaMemcpy(h.data(), counts, sizeof(int64_t) * h.size(), cudaMemcpyDeviceToHost));
    for (int x = 0; x < NCLS; ++x)
        for (int y = 0; y < NCLS; ++y) {
            int64_t t = 0;
            if (y <= x)
                for (int sub = 0; sub < NSUB; ++sub)
                    for (int s = c->cls_start[x]; s < c->cls_start[x + 1]; ++s) t += h[(size_t)(y * NSUB + sub) * n + s];
            out_host[x * NCLS + y] = t;
        }
    return AIMD_OK;
}

extern "C" int aimd_pair_data(aimd_ctx* c, int* npp_host, int* cls_host, int* sorted_host) {
    // per pair: surviving primitive pairs; per sorted position: class and pair index
    if (!c || !c->have_geometry) return AIMD_ERR_ARG;
    if (npp_host) CK(cudaMemcpy(npp_host, c->npp, sizeof(int) * c->npair, cudaMemcpyDeviceToHost));
    if (sorted_host) CK(cudaMemcpy(sorted_host, c->sorted, sizeof(int) * c->npair, cudaMemcpyDeviceToHost));
    if (cls_host)
        for (int cl = 0; cl < NCLS; ++cl)
            for (int s = c->cls_start[cl]; s < c->cls_start[cl + 1]; ++s) cls_host[s] = cl;
    return AIMD_OK;
}

extern "C" uint64_t aimd_launch_count(aimd_ctx* c) { return c ? c->launches : 0; }

extern "C" int aimd_sizes(aimd_ctx* c, int* natm, int* nao) {
    if (!c || !natm || !nao) return AIMD_ERR_ARG;
    *natm = c->natm;
    *nao = c->nao;
    return AIMD_OK;
}

// sum_{A<B} Z_A Z_B / |R_A - R_B| of the current geometry (host value; the
// positions are read back on `stream`, after the aimd_set_geometry that set
// them)
extern "C" int aimd_nuclear_repulsion(aimd_ctx* c, double* energy, void* stream) {
    if (!c || !energy || !c->have_geometry) return AIMD_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<double> x(3 * (size_t)c->natm);
    CK(cudaMemcpyAsync(x.data(), c->pos, sizeof(double) * x.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double e = 0.0;
    for (int a = 0; a < c->natm; ++a)
        for (int b = 0; b < a; ++b) {
            const double dx = x[3 * a] - x[3 * b], dy = x[3 * a + 1] - x[3 * b + 1], dz = x[3 * a + 2] - x[3 * b + 2];
            e += c->charges_host[a] * c->charges_host[b] / sqrt(dx * dx + dy * dy + dz * dz);
        }
    *energy = e;
    return AIMD_OK;
}

extern "C" int aimd_version(void) { return AIMD_ABI_VERSION; }
