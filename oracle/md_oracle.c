/*
 * ORACLE (test infrastructure only): CPU restatement of the reference's
 * McMurchie-Davidson integral path (Nathan-W123/Ab-Initio-MD, aimd/qc).
 *
 * This file is the checker for the CUDA product path. Only tests/, the
 * smoke() entry and bench.py's CPU-baseline leg load it. Parity of this
 * restatement with the reference itself is pinned by the golden fixtures in
 * tests/golden (generated by importing the reference, see
 * tests/golden/make_golden.py).
 *
 * Every function follows one reference function; the file:line is given
 * beside it. Threading: OpenMP over bra block pairs, per-thread
 * accumulators summed in thread order at the end.
 *
 * Build: oracle/Makefile  ->  oracle/_build/libmd_oracle.so
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LMAX 4                      /* aimd/qc/hermite.py:51 */
#define HMAX (4 * LMAX + 1)         /* aimd/qc/hermite.py:52 */
#define NHTOT ((HMAX + 1) * (HMAX + 2) * (HMAX + 3) / 6)
#define BOYS_NMAX 32                /* aimd/qc/boys.py:49-54 */
#define BOYS_NTAYLOR 10
#define BOYS_STEP 0.1
#define BOYS_SWITCH 40.0
#define BOYS_NGRID 402
#define BOYS_NROWS (BOYS_NMAX + BOYS_NTAYLOR + 1)
#define PRIM_CUTOFF 50.0            /* aimd/qc/integrals.py:510 */

typedef int64_t i64;

static double boys_table[BOYS_NGRID][BOYS_NROWS];
static double inv_odd[BOYS_NMAX + 1];
static double inv_int[BOYS_NTAYLOR];
static int herm_tuv[NHTOT][3];
static int herm_idx[HMAX + 2][HMAX + 2][HMAX + 2];
static int herm_dir[NHTOT], herm_m1[NHTOT], herm_m2[NHTOT];
static double herm_rc[NHTOT], herm_sign[NHTOT];
static int nherm_tab[HMAX + 2];
static int cart_off[LMAX + 3];
static int cart_lxyz[64][3];
static double cart_fac[64];
static int ready = 0;

static const double PI = 3.14159265358979323846;

static int nh(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

static i64 dfact(int n) { i64 r = 1; while (n > 1) { r *= n; n -= 2; } return r; }

/* boys.py:57-79 (grid table by the positive series for the top order, then
 * downward recursion), hermite.py:59-105 (Cartesian and Hermite tables). */
static void init_tables(void) {
    if (ready) return;
    int top = BOYS_NROWS - 1;
    for (int k = 0; k < BOYS_NGRID; k++) {
        double x = k * BOYS_STEP;
        double term = 1.0 / (2 * top + 1), total = term;
        for (int j = 1; j < 400; j++) { term = term * (2.0 * x) / (2 * top + 2 * j + 1); total += term; }
        double ex = exp(-x);
        boys_table[k][top] = ex * total;
        for (int n = top - 1; n >= 0; n--)
            boys_table[k][n] = (2.0 * x * boys_table[k][n + 1] + ex) / (2 * n + 1);
    }
    for (int n = 0; n <= BOYS_NMAX; n++) inv_odd[n] = 1.0 / (2 * n + 1);
    for (int m = 0; m < BOYS_NTAYLOR; m++) inv_int[m] = 1.0 / (m + 1);
    int h = 0;
    for (int d = 0; d <= HMAX; d++)
        for (int t = d; t >= 0; t--)
            for (int u = d - t; u >= 0; u--) {
                herm_tuv[h][0] = t; herm_tuv[h][1] = u; herm_tuv[h][2] = d - t - u; h++;
            }
    for (int a = 0; a < HMAX + 2; a++)
        for (int b = 0; b < HMAX + 2; b++)
            for (int c = 0; c < HMAX + 2; c++) herm_idx[a][b][c] = -1;
    for (int i = 0; i < NHTOT; i++) herm_idx[herm_tuv[i][0]][herm_tuv[i][1]][herm_tuv[i][2]] = i;
    for (int i = 0; i < NHTOT; i++) {
        herm_dir[i] = herm_m1[i] = herm_m2[i] = 0; herm_rc[i] = 0.0;
        int c[3] = {herm_tuv[i][0], herm_tuv[i][1], herm_tuv[i][2]};
        herm_sign[i] = ((c[0] + c[1] + c[2]) % 2 == 0) ? 1.0 : -1.0;
        if (i == 0) continue;
        int d = c[0] > 0 ? 0 : (c[1] > 0 ? 1 : 2);
        herm_dir[i] = d;
        int c1[3] = {c[0], c[1], c[2]}; c1[d] -= 1;
        herm_m1[i] = herm_idx[c1[0]][c1[1]][c1[2]];
        if (c[d] >= 2) {
            int c2[3] = {c[0], c[1], c[2]}; c2[d] -= 2;
            herm_m2[i] = herm_idx[c2[0]][c2[1]][c2[2]];
            herm_rc[i] = c[d] - 1;
        }
    }
    for (int L = 0; L < HMAX + 2; L++) nherm_tab[L] = nh(L);
    int n = 0;
    cart_off[0] = 0;
    for (int l = 0; l <= LMAX + 1; l++) {
        for (int lx = l; lx >= 0; lx--)
            for (int ly = l - lx; ly >= 0; ly--) {
                int lz = l - lx - ly;
                cart_lxyz[n][0] = lx; cart_lxyz[n][1] = ly; cart_lxyz[n][2] = lz;
                cart_fac[n] = sqrt((double)dfact(2 * l - 1) /
                                   (double)(dfact(2 * lx - 1) * dfact(2 * ly - 1) * dfact(2 * lz - 1)));
                n++;
            }
        cart_off[l + 1] = n;
    }
    ready = 1;
}

/* boys.py:88-114 */
static double boys_top(int n, double x) {
    if (x < BOYS_SWITCH) {
        int k = (int)(x * (1.0 / BOYS_STEP) + 0.5);
        double dx = k * BOYS_STEP - x, acc = 0.0, fac = 1.0;
        for (int m = 0; m < BOYS_NTAYLOR; m++) { acc += boys_table[k][n + m] * fac; fac *= dx * inv_int[m]; }
        return acc;
    }
    double f = 0.5 * sqrt(PI / x);
    if (n > 0) {
        double ex = exp(-x), inv2x = 0.5 / x;
        for (int m = 0; m < n; m++) f = ((2 * m + 1) * f - ex) * inv2x;
    }
    return f;
}

/* boys.py:118-140 */
void orc_boys(int nmax, double x, double *out) {
    init_tables();
    if (x >= BOYS_SWITCH) {
        double f = 0.5 * sqrt(PI / x), ex = exp(-x), inv2x = 0.5 / x;
        out[0] = f;
        for (int n = 0; n < nmax; n++) { f = ((2 * n + 1) * f - ex) * inv2x; out[n + 1] = f; }
        return;
    }
    double f = boys_top(nmax, x);
    out[nmax] = f;
    double ex = exp(-x), x2 = 2.0 * x;
    for (int n = nmax - 1; n >= 0; n--) { f = (x2 * f + ex) * inv_odd[n]; out[n] = f; }
}

/* E layout: e[(i * sj + j) * st + t] */
/* hermite.py:110-141 */
static void hermite_e(int imax, int jmax, double a, double b, double xab, double e00,
                      double *e, int sj, int st) {
    double p = a + b, xpa = -b * xab / p, xpb = a * xab / p, hh = 0.5 / p;
    int tmax = imax + jmax + 1;
    for (int i = 0; i <= imax; i++)
        for (int j = 0; j <= jmax; j++)
            for (int t = 0; t <= tmax; t++) e[(i * sj + j) * st + t] = 0.0;
    e[0] = e00;
    for (int j = 1; j <= jmax; j++)
        for (int t = 0; t <= j; t++) {
            double v = xpb * e[(0 * sj + j - 1) * st + t] + (t + 1) * e[(0 * sj + j - 1) * st + t + 1];
            if (t > 0) v += hh * e[(0 * sj + j - 1) * st + t - 1];
            e[(0 * sj + j) * st + t] = v;
        }
    for (int i = 1; i <= imax; i++)
        for (int j = 0; j <= jmax; j++)
            for (int t = 0; t <= i + j; t++) {
                double v = xpa * e[((i - 1) * sj + j) * st + t] + (t + 1) * e[((i - 1) * sj + j) * st + t + 1];
                if (t > 0) v += hh * e[((i - 1) * sj + j) * st + t - 1];
                e[(i * sj + j) * st + t] = v;
            }
}

/* hermite.py:145-178 and its inlined copies integrals.py:723-746:
 * out[h] = R_tuv(alpha, x, y, z), h < NH(L). tmp: scratch of NH(L). */
static void hermite_r(int L, double alpha, double x, double y, double z, double *out, double *tmp) {
    double T = alpha * (x * x + y * y + z * z);
    double f = boys_top(L, T);
    double ex = L > 0 ? exp(-T) : 0.0;
    double t2 = 2.0 * T, m2a = -2.0 * alpha, pw = 1.0;
    double xyz[3] = {x, y, z};
    for (int i = 0; i < L; i++) pw *= m2a;
    for (int n = L; n >= 0; n--) {
        if (n < L) f = (t2 * f + ex) * inv_odd[n];
        double *cur = (n % 2 == 0) ? out : tmp;
        double *prv = (n % 2 == 0) ? tmp : out;
        cur[0] = pw * f;
        for (int h = 1; h < nherm_tab[L - n]; h++)
            cur[h] = xyz[herm_dir[h]] * prv[herm_m1[h]] + herm_rc[h] * prv[herm_m2[h]];
        pw /= m2a;
    }
}

/* ===================================================== block pairs */

/* Dimensions of the pair arrays for a basis with maximum l = lmax. */
static int E_L1(int lmax) { return lmax + 2; }
static int E_T1(int lmax) { return 2 * lmax + 4; }

/* integrals.py:525-599 (_build_pairs). Count pass: returns npp and fills
 * pair_pp (npair + 1) and pair_blocks (npair x 2). */
i64 orc_count_pairs(i64 nb, const i64 *blk_atom, const i64 *blk_prim, const double *blk_exp,
                    const double *pos, i64 *pair_pp, i64 *pair_blocks) {
    i64 npp = 0, ip = 0;
    for (i64 i = 0; i < nb; i++)
        for (i64 j = 0; j <= i; j++) {
            pair_pp[ip] = npp; pair_blocks[2 * ip] = i; pair_blocks[2 * ip + 1] = j;
            double r2 = 0.0;
            for (int d = 0; d < 3; d++) {
                double dx = pos[3 * blk_atom[i] + d] - pos[3 * blk_atom[j] + d]; r2 += dx * dx;
            }
            for (i64 ka = blk_prim[i]; ka < blk_prim[i + 1]; ka++)
                for (i64 kb = blk_prim[j]; kb < blk_prim[j + 1]; kb++) {
                    double a = blk_exp[ka], b = blk_exp[kb];
                    if (a * b / (a + b) * r2 <= PRIM_CUTOFF) npp++;
                }
            ip++;
        }
    pair_pp[ip] = npp;
    return npp;
}

/* Fill pass of _build_pairs: pp_ab[npp,2], pp_P[npp,3], pp_E[npp,3,L1,L1,T1],
 * pp_C[npp, maxcon^2]. */
void orc_fill_pairs(i64 nb, i64 lmax, i64 maxcon, const i64 *blk_atom, const i64 *blk_l,
                    const i64 *blk_prim, const double *blk_exp, const double *blk_coef,
                    const i64 *blk_ncon, const double *pos, double *pp_ab, double *pp_P,
                    double *pp_E, double *pp_C) {
    init_tables();
    int L1 = E_L1(lmax), T1 = E_T1(lmax);
    i64 k = 0;
    for (i64 i = 0; i < nb; i++) {
        i64 ai = blk_atom[i];
        for (i64 j = 0; j <= i; j++) {
            i64 aj = blk_atom[j], ncj = blk_ncon[j];
            double r2 = 0.0;
            for (int d = 0; d < 3; d++) { double dx = pos[3 * ai + d] - pos[3 * aj + d]; r2 += dx * dx; }
            for (i64 ka = blk_prim[i]; ka < blk_prim[i + 1]; ka++) {
                double a = blk_exp[ka];
                for (i64 kb = blk_prim[j]; kb < blk_prim[j + 1]; kb++) {
                    double b = blk_exp[kb], p = a + b, mu = a * b / p;
                    if (!(mu * r2 <= PRIM_CUTOFF)) continue;
                    pp_ab[2 * k] = a; pp_ab[2 * k + 1] = b;
                    for (i64 ci = 0; ci < blk_ncon[i]; ci++)
                        for (i64 cj = 0; cj < ncj; cj++)
                            pp_C[k * maxcon * maxcon + ci * ncj + cj] =
                                blk_coef[ka * maxcon + ci] * blk_coef[kb * maxcon + cj];
                    for (int d = 0; d < 3; d++) {
                        double xab = pos[3 * ai + d] - pos[3 * aj + d];
                        pp_P[3 * k + d] = pos[3 * ai + d] - (b / p) * xab;
                        hermite_e((int)blk_l[i] + 1, (int)blk_l[j] + 1, a, b, xab, exp(-mu * xab * xab),
                                  pp_E + ((k * 3 + d) * L1 * L1) * T1, L1, T1);
                    }
                    k++;
                }
            }
        }
    }
}

/* Everything an ERI block evaluation needs about the basis and its pairs. */
typedef struct {
    i64 nb, npair, npp, lmax, maxcon, maxpp, maxrow;
    const i64 *blk_l, *blk_ncon, *blk_ao, *blk_atom;
    const i64 *pair_pp, *pair_blocks;
    const double *pp_ab, *pp_P, *pp_E, *pp_C;
} Pairs;

typedef struct {
    double *block, *Ek, *X, *T, *W, *RR, *Gb;
    int *hidx;
    i64 ekk, ekc, xc, hidc;   /* row strides */
} Scratch;

#define PE(pr, k, d, i, j, t) \
    (pr)->pp_E[((((k) * 3 + (d)) * E_L1((pr)->lmax) + (i)) * E_L1((pr)->lmax) + (j)) * E_T1((pr)->lmax) + (t)]

static void pair_dims(const Pairs *pr, i64 ip, int *nab, int *nbc) {
    i64 i = pr->pair_blocks[2 * ip], j = pr->pair_blocks[2 * ip + 1];
    int li = (int)pr->blk_l[i], lj = (int)pr->blk_l[j];
    *nab = (cart_off[li + 1] - cart_off[li]) * (cart_off[lj + 1] - cart_off[lj]);
    *nbc = (int)(pr->blk_ncon[i] * pr->blk_ncon[j]);
}

static Scratch scratch_new(const Pairs *pr, int deriv) {
    Scratch s;
    int lmax = (int)pr->lmax, nc = (lmax + 1) * (lmax + 2) / 2;
    i64 nhp = nh(2 * lmax + deriv), nR = nh(4 * lmax + deriv), nhk = nh(2 * lmax);
    s.ekk = nhk; s.ekc = nc * nc; s.xc = pr->maxrow; s.hidc = nhk;
    s.block = malloc(sizeof(double) * pr->maxrow * pr->maxrow);
    s.Ek = malloc(sizeof(double) * pr->maxpp * nhk * nc * nc);
    s.X = malloc(sizeof(double) * nhp * pr->maxrow);
    s.T = malloc(sizeof(double) * nc * nc);
    s.W = malloc(sizeof(double) * nc * nc * pr->maxrow);
    s.Gb = malloc(sizeof(double) * nc * nc * pr->maxrow);
    s.RR = malloc(sizeof(double) * 2 * nR);
    s.hidx = malloc(sizeof(int) * nhp * nhk);
    return s;
}

static void scratch_free(Scratch *s) {
    free(s->block); free(s->Ek); free(s->X); free(s->T); free(s->W); free(s->Gb); free(s->RR); free(s->hidx);
}

/* integrals.py:646-682 (_ket_hermite) */
static void ket_hermite(const Pairs *pr, i64 pk, Scratch *s) {
    i64 sk = pr->pair_blocks[2 * pk], sl = pr->pair_blocks[2 * pk + 1];
    int lk = (int)pr->blk_l[sk], ll = (int)pr->blk_l[sl];
    int c0 = cart_off[lk], nck = cart_off[lk + 1] - c0, d0 = cart_off[ll], ncl = cart_off[ll + 1] - d0;
    int nhk = nh(lk + ll);
    i64 k0 = pr->pair_pp[pk];
    for (i64 kp = 0; kp < pr->pair_pp[pk + 1] - k0; kp++) {
        double *Ek = s->Ek + kp * s->ekk * s->ekc;
        for (int k = 0; k < nhk; k++)
            for (int cd = 0; cd < nck * ncl; cd++) Ek[k * s->ekc + cd] = 0.0;
        for (int ic = 0; ic < nck; ic++) {
            int cx = cart_lxyz[c0 + ic][0], cy = cart_lxyz[c0 + ic][1], cz = cart_lxyz[c0 + ic][2];
            for (int id = 0; id < ncl; id++) {
                int dx = cart_lxyz[d0 + id][0], dy = cart_lxyz[d0 + id][1], dz = cart_lxyz[d0 + id][2];
                double f = cart_fac[c0 + ic] * cart_fac[d0 + id];
                int cd = ic * ncl + id;
                for (int t = 0; t <= cx + dx; t++) {
                    double et = f * PE(pr, k0 + kp, 0, cx, dx, t);
                    for (int u = 0; u <= cy + dy; u++) {
                        double etu = et * PE(pr, k0 + kp, 1, cy, dy, u);
                        for (int v = 0; v <= cz + dz; v++) {
                            int kk = herm_idx[t][u][v];
                            Ek[kk * s->ekc + cd] = herm_sign[kk] * etu * PE(pr, k0 + kp, 2, cz, dz, v);
                        }
                    }
                }
            }
        }
    }
}

/* integrals.py:685-690 (_hidx_fill) */
static void hidx_fill(int nhb, int nhk, Scratch *s) {
    for (int h = 0; h < nhb; h++)
        for (int k = 0; k < nhk; k++)
            s->hidx[h * s->hidc + k] = herm_idx[herm_tuv[h][0] + herm_tuv[k][0]][herm_tuv[h][1] + herm_tuv[k][1]]
                                               [herm_tuv[h][2] + herm_tuv[k][2]];
}

/* integrals.py:705-774 (_ket_r_contract): X[h, ckl*ncd + cd] for bra prim pair bp */
static void ket_r_contract(const Pairs *pr, i64 bp, i64 pk, int nhb, int L, int nhk, int ncd, int nkc,
                           Scratch *s) {
    const double two_pi_2_5 = 2.0 * pow(PI, 2.5);
    double p = pr->pp_ab[2 * bp] + pr->pp_ab[2 * bp + 1];
    int ncol = nkc * ncd;
    for (int h = 0; h < nhb; h++)
        for (int c = 0; c < ncol; c++) s->X[h * s->xc + c] = 0.0;
    i64 k0 = pr->pair_pp[pk];
    double *R = s->RR, *tmp = s->RR + nh(L);
    for (i64 kp = 0; kp < pr->pair_pp[pk + 1] - k0; kp++) {
        i64 kq = k0 + kp;
        double q = pr->pp_ab[2 * kq] + pr->pp_ab[2 * kq + 1];
        double alpha = p * q / (p + q), pref = two_pi_2_5 / (p * q * sqrt(p + q));
        hermite_r(L, alpha, pr->pp_P[3 * bp] - pr->pp_P[3 * kq], pr->pp_P[3 * bp + 1] - pr->pp_P[3 * kq + 1],
                  pr->pp_P[3 * bp + 2] - pr->pp_P[3 * kq + 2], R, tmp);
        const double *Ek = s->Ek + kp * s->ekk * s->ekc;
        for (int h = 0; h < nhb; h++) {
            for (int cd = 0; cd < ncd; cd++) s->T[cd] = 0.0;
            for (int k = 0; k < nhk; k++) {
                double r = pref * R[s->hidx[h * s->hidc + k]];
                if (r == 0.0) continue;
                for (int cd = 0; cd < ncd; cd++) s->T[cd] += r * Ek[k * s->ekc + cd];
            }
            for (int ckl = 0; ckl < nkc; ckl++) {
                double c = pr->pp_C[kq * pr->maxcon * pr->maxcon + ckl];
                if (c == 0.0) continue;
                for (int cd = 0; cd < ncd; cd++) s->X[h * s->xc + ckl * ncd + cd] += c * s->T[cd];
            }
        }
    }
}

/* integrals.py:777-842 (_eri_block): block[r, c] = (IJ|KL), row/col layout of the reference */
static void eri_block(const Pairs *pr, i64 pb, i64 pk, Scratch *s) {
    i64 si = pr->pair_blocks[2 * pb], sj = pr->pair_blocks[2 * pb + 1];
    i64 sk = pr->pair_blocks[2 * pk], sl = pr->pair_blocks[2 * pk + 1];
    int li = (int)pr->blk_l[si], lj = (int)pr->blk_l[sj];
    int a0 = cart_off[li], nci = cart_off[li + 1] - a0, b0 = cart_off[lj], ncj = cart_off[lj + 1] - b0;
    int nab, nbc, ncd, nkc;
    pair_dims(pr, pb, &nab, &nbc);
    pair_dims(pr, pk, &ncd, &nkc);
    int ncol = nkc * ncd, Lab = li + lj;
    int L = Lab + (int)pr->blk_l[sk] + (int)pr->blk_l[sl];
    int nhb = nh(Lab), nhk = nh((int)(pr->blk_l[sk] + pr->blk_l[sl]));
    hidx_fill(nhb, nhk, s);
    ket_hermite(pr, pk, s);
    i64 mr = pr->maxrow;
    for (int r = 0; r < nbc * nab; r++)
        for (int c = 0; c < ncol; c++) s->block[r * mr + c] = 0.0;
    for (i64 bp = pr->pair_pp[pb]; bp < pr->pair_pp[pb + 1]; bp++) {
        ket_r_contract(pr, bp, pk, nhb, L, nhk, ncd, nkc, s);
        double cb = nbc == 1 ? pr->pp_C[bp * pr->maxcon * pr->maxcon] : 1.0;
        for (int ia = 0; ia < nci; ia++) {
            int ax = cart_lxyz[a0 + ia][0], ay = cart_lxyz[a0 + ia][1], az = cart_lxyz[a0 + ia][2];
            double fa = cb * cart_fac[a0 + ia];
            for (int ib = 0; ib < ncj; ib++) {
                int bx = cart_lxyz[b0 + ib][0], by = cart_lxyz[b0 + ib][1], bz = cart_lxyz[b0 + ib][2];
                double f = fa * cart_fac[b0 + ib];
                int ab = ia * ncj + ib;
                double *out = nbc == 1 ? s->block + ab * mr : s->W + ab * mr;
                if (nbc != 1)
                    for (int c = 0; c < ncol; c++) out[c] = 0.0;
                for (int t = 0; t <= ax + bx; t++) {
                    double et = f * PE(pr, bp, 0, ax, bx, t);
                    for (int u = 0; u <= ay + by; u++) {
                        double etu = et * PE(pr, bp, 1, ay, by, u);
                        for (int v = 0; v <= az + bz; v++) {
                            double e = etu * PE(pr, bp, 2, az, bz, v);
                            int h = herm_idx[t][u][v];
                            for (int c = 0; c < ncol; c++) out[c] += e * s->X[h * s->xc + c];
                        }
                    }
                }
            }
        }
        if (nbc != 1)
            for (int cij = 0; cij < nbc; cij++) {
                double c = pr->pp_C[bp * pr->maxcon * pr->maxcon + cij];
                if (c == 0.0) continue;
                for (int ab = 0; ab < nab; ab++)
                    for (int col = 0; col < ncol; col++)
                        s->block[(cij * nab + ab) * mr + col] += c * s->W[ab * mr + col];
            }
    }
}

static Pairs make_pairs(i64 nb, i64 npp, i64 lmax, i64 maxcon, i64 maxpp, i64 maxrow, const i64 *blk_l,
                        const i64 *blk_ncon, const i64 *blk_ao, const i64 *blk_atom, const i64 *pair_pp,
                        const i64 *pair_blocks, const double *pp_ab, const double *pp_P, const double *pp_E,
                        const double *pp_C) {
    Pairs p;
    p.nb = nb; p.npair = nb * (nb + 1) / 2; p.npp = npp; p.lmax = lmax; p.maxcon = maxcon;
    p.maxpp = maxpp; p.maxrow = maxrow; p.blk_l = blk_l; p.blk_ncon = blk_ncon; p.blk_ao = blk_ao;
    p.blk_atom = blk_atom; p.pair_pp = pair_pp; p.pair_blocks = pair_blocks; p.pp_ab = pp_ab;
    p.pp_P = pp_P; p.pp_E = pp_E; p.pp_C = pp_C;
    return p;
}

#define PAIR_ARGS i64 nb, i64 npp, i64 lmax, i64 maxcon, i64 maxpp, i64 maxrow, const i64 *blk_l, \
    const i64 *blk_ncon, const i64 *blk_ao, const i64 *blk_atom, const i64 *pair_pp, const i64 *pair_blocks, \
    const double *pp_ab, const double *pp_P, const double *pp_E, const double *pp_C
#define PAIR_PASS nb, npp, lmax, maxcon, maxpp, maxrow, blk_l, blk_ncon, blk_ao, blk_atom, pair_pp, \
    pair_blocks, pp_ab, pp_P, pp_E, pp_C

/* integrals.py:864-883 (_schwarz_kernel) */
void orc_schwarz(PAIR_ARGS, double *Q) {
    init_tables();
    Pairs pr = make_pairs(PAIR_PASS);
#pragma omp parallel
    {
        Scratch s = scratch_new(&pr, 0);
#pragma omp for schedule(dynamic, 1)
        for (i64 ip = 0; ip < pr.npair; ip++) {
            eri_block(&pr, ip, ip, &s);
            int nab, nbc;
            pair_dims(&pr, ip, &nab, &nbc);
            double m = 0.0;
            for (int r = 0; r < nab * nbc; r++) m = fmax(m, fabs(s.block[r * pr.maxrow + r]));
            Q[ip] = sqrt(m);
        }
        scratch_free(&s);
    }
}

/* Visit the elements of one unique block quartet (p1 >= p2) in the
 * reference's orientation: v = (m n | l s) with m in I, n in J, l in K,
 * s in L; the block was computed with the smaller pair in the ket
 * (integrals.py:900-915) and is read back transposed when swapped. */
#define QUARTET_LOOP(pr, p1, p2, swapped, s, ...) do { \
    i64 si_ = (pr)->pair_blocks[2 * (p1)], sj_ = (pr)->pair_blocks[2 * (p1) + 1]; \
    i64 sk_ = (pr)->pair_blocks[2 * (p2)], sl_ = (pr)->pair_blocks[2 * (p2) + 1]; \
    int nci_ = cart_off[(pr)->blk_l[si_] + 1] - cart_off[(pr)->blk_l[si_]]; \
    int ncj_ = cart_off[(pr)->blk_l[sj_] + 1] - cart_off[(pr)->blk_l[sj_]]; \
    int nck_ = cart_off[(pr)->blk_l[sk_] + 1] - cart_off[(pr)->blk_l[sk_]]; \
    int ncl_ = cart_off[(pr)->blk_l[sl_] + 1] - cart_off[(pr)->blk_l[sl_]]; \
    int n1_ = nci_ * ncj_, n2_ = nck_ * ncl_; \
    i64 nqj_ = (pr)->blk_ncon[sj_], nql_ = (pr)->blk_ncon[sl_]; \
    for (i64 qi = 0; qi < (pr)->blk_ncon[si_]; qi++) for (int a_ = 0; a_ < nci_; a_++) { \
        i64 m = (pr)->blk_ao[si_] + qi * nci_ + a_; \
        for (i64 qj = 0; qj < nqj_; qj++) for (int b_ = 0; b_ < ncj_; b_++) { \
            i64 n = (pr)->blk_ao[sj_] + qj * ncj_ + b_; \
            i64 r1_ = (qi * nqj_ + qj) * n1_ + a_ * ncj_ + b_; \
            for (i64 qk = 0; qk < (pr)->blk_ncon[sk_]; qk++) for (int c_ = 0; c_ < nck_; c_++) { \
                i64 l = (pr)->blk_ao[sk_] + qk * nck_ + c_; \
                for (i64 ql = 0; ql < nql_; ql++) for (int d_ = 0; d_ < ncl_; d_++) { \
                    i64 sg = (pr)->blk_ao[sl_] + ql * ncl_ + d_; \
                    i64 r2_ = (qk * nql_ + ql) * n2_ + c_ * ncl_ + d_; \
                    double v = (swapped) ? (s)->block[r2_ * (pr)->maxrow + r1_] : (s)->block[r1_ * (pr)->maxrow + r2_]; \
                    __VA_ARGS__ \
                } } } } } while (0)

static int quartet_swapped(const Pairs *pr, i64 p1, i64 p2) {
    int n1, c1, n2, c2;
    pair_dims(pr, p1, &n1, &c1);
    pair_dims(pr, p2, &n2, &c2);
    return n1 * c1 < n2 * c2;
}

/* integrals.py:886-949 (_eri_tensor_kernel) + :952-967 (_symmetrize_pairs):
 * full tensor, nao^4 doubles (test sizes only). */
void orc_eri_tensor(PAIR_ARGS, const double *Q, double threshold, i64 nao, double *eri) {
    init_tables();
    Pairs pr = make_pairs(PAIR_PASS);
    i64 N = nao, n2 = nao * nao, n3 = n2 * nao;
#pragma omp parallel
    {
        Scratch s = scratch_new(&pr, 0);
#pragma omp for schedule(dynamic, 1)
        for (i64 p1 = 0; p1 < pr.npair; p1++)
            for (i64 p2 = 0; p2 <= p1; p2++) {
                if (Q[p1] * Q[p2] < threshold) continue;
                int sw = quartet_swapped(&pr, p1, p2);
                if (sw) eri_block(&pr, p2, p1, &s); else eri_block(&pr, p1, p2, &s);
                double scale = p1 == p2 ? 0.5 : 1.0;
                QUARTET_LOOP(&pr, p1, p2, sw, &s, {
                    double w = scale * v;
                    eri[m * n3 + n * n2 + l * N + sg] = w;
                    eri[n * n3 + m * n2 + l * N + sg] = w;
                    eri[m * n3 + n * n2 + sg * N + l] = w;
                    eri[n * n3 + m * n2 + sg * N + l] = w;
                });
            }
        scratch_free(&s);
    }
    for (i64 r = 0; r < n2; r++)
        for (i64 c = 0; c <= r; c++) {
            double v = eri[r * n2 + c] + eri[c * n2 + r];
            eri[r * n2 + c] = v; eri[c * n2 + r] = v;
        }
}

/* Integral-direct J/K over the same unique, Schwarz-screened block quartets
 * as integrals.py:900-915, digested with the 8-fold index map of
 * integrals.py:928-949 (each tensor element visited 1/n_gen times) instead
 * of being stored. Outputs are the un-symmetrised accumulators
 *   Jacc[s, m, n] += 2 g v D[s, l, sg], Jacc[s, l, sg] += 2 g v D[s, m, n]
 *   Kacc[s, m, l] += g v D[s, n, sg]  (and the three other exchange images)
 * with g = 1 / n_gen, n_gen = the number of times the block visits each
 * tensor element under the 8 index maps; J = Jacc + Jacc^T and, for symmetric D, K = Kacc + Kacc^T
 * (reference result jk_from_eri(eri_tensor, D), integrals.py:1009-1044). */
/* Bra pairs p1 with p1 % stride == offset only (stride 1: the whole build);
 * the bench times strided samples of one build on the host cores. */
void orc_jk_direct_strided(PAIR_ARGS, const double *Q, double threshold, i64 nao, i64 nset, const double *D,
                           double *Jacc, double *Kacc, i64 stride, i64 offset);

void orc_jk_direct(PAIR_ARGS, const double *Q, double threshold, i64 nao, i64 nset, const double *D,
                   double *Jacc, double *Kacc) {
    orc_jk_direct_strided(PAIR_PASS, Q, threshold, nao, nset, D, Jacc, Kacc, 1, 0);
}

void orc_jk_direct_strided(PAIR_ARGS, const double *Q, double threshold, i64 nao, i64 nset, const double *D,
                           double *Jacc, double *Kacc, i64 stride, i64 offset) {
    init_tables();
    Pairs pr = make_pairs(PAIR_PASS);
    i64 n2 = nao * nao, tot = nset * n2;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    double *acc = calloc((size_t)nthr * 2 * tot, sizeof(double));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *J = acc + (size_t)tid * 2 * tot, *K = J + tot;
        Scratch s = scratch_new(&pr, 0);
#pragma omp for schedule(dynamic, 1)
        for (i64 p1 = offset; p1 < pr.npair; p1 += stride)
            for (i64 p2 = 0; p2 <= p1; p2++) {
                if (Q[p1] * Q[p2] < threshold) continue;
                int sw = quartet_swapped(&pr, p1, p2);
                if (sw) eri_block(&pr, p2, p1, &s); else eri_block(&pr, p1, p2, &s);
                i64 I = pr.pair_blocks[2 * p1], Jb = pr.pair_blocks[2 * p1 + 1];
                i64 K_ = pr.pair_blocks[2 * p2], L_ = pr.pair_blocks[2 * p2 + 1];
                double ngen = (I == Jb ? 2.0 : 1.0) * (K_ == L_ ? 2.0 : 1.0) * (p1 == p2 ? 2.0 : 1.0);
                double g = 1.0 / ngen;
                QUARTET_LOOP(&pr, p1, p2, sw, &s, {
                    double gv = g * v;
                    for (i64 st = 0; st < nset; st++) {
                        const double *Ds = D + st * n2;
                        double *Js = J + st * n2, *Ks = K + st * n2;
                        Js[m * nao + n] += 2.0 * gv * Ds[l * nao + sg];
                        Js[l * nao + sg] += 2.0 * gv * Ds[m * nao + n];
                        Ks[m * nao + l] += gv * Ds[n * nao + sg];
                        Ks[n * nao + l] += gv * Ds[m * nao + sg];
                        Ks[m * nao + sg] += gv * Ds[n * nao + l];
                        Ks[n * nao + sg] += gv * Ds[m * nao + l];
                    }
                });
            }
        scratch_free(&s);
    }
    for (i64 i = 0; i < tot; i++) {
        double sj = 0.0, sk = 0.0;
        for (int t = 0; t < nthr; t++) { sj += acc[(size_t)t * 2 * tot + i]; sk += acc[(size_t)t * 2 * tot + tot + i]; }
        Jacc[i] = sj; Kacc[i] = sk;
    }
    free(acc);
}

/* integrals.py:1049-1244 (_grad_pass), the post-R ("use_x") contraction order
 * for every quartet: out[0..2] = d/dA, out[3..5] = d/dB of sum G (IJ|KL). */
static void grad_pass(const Pairs *pr, i64 pb, i64 pk, const double *G, i64 gs, Scratch *s, double *out) {
    i64 si = pr->pair_blocks[2 * pb], sj = pr->pair_blocks[2 * pb + 1];
    i64 sk = pr->pair_blocks[2 * pk], sl = pr->pair_blocks[2 * pk + 1];
    int li = (int)pr->blk_l[si], lj = (int)pr->blk_l[sj], lk = (int)pr->blk_l[sk], ll = (int)pr->blk_l[sl];
    int a0 = cart_off[li], nci = cart_off[li + 1] - a0, b0 = cart_off[lj], ncj = cart_off[lj + 1] - b0;
    int nab, nbc, ncd, nkc;
    pair_dims(pr, pb, &nab, &nbc);
    pair_dims(pr, pk, &ncd, &nkc);
    int ncol = nkc * ncd, Lab = li + lj, L = Lab + lk + ll + 1;
    int nh1 = nh(Lab + 1), nhk = nh(lk + ll);
    hidx_fill(nh1, nhk, s);
    ket_hermite(pr, pk, s);
    for (int d = 0; d < 6; d++) out[d] = 0.0;
    i64 mr = pr->maxrow;
    for (i64 bp = pr->pair_pp[pb]; bp < pr->pair_pp[pb + 1]; bp++) {
        double a = pr->pp_ab[2 * bp], b = pr->pp_ab[2 * bp + 1];
        double cb = nbc == 1 ? pr->pp_C[bp * pr->maxcon * pr->maxcon] : 1.0;
        ket_r_contract(pr, bp, pk, nh1, L, nhk, ncd, nkc, s);
        if (nbc != 1) {
            for (int ab = 0; ab < nab; ab++)
                for (int c = 0; c < ncol; c++) s->Gb[ab * mr + c] = 0.0;
            for (int cij = 0; cij < nbc; cij++) {
                double c = pr->pp_C[bp * pr->maxcon * pr->maxcon + cij];
                if (c == 0.0) continue;
                for (int ab = 0; ab < nab; ab++)
                    for (int col = 0; col < ncol; col++) s->Gb[ab * mr + col] += c * G[(cij * nab + ab) * gs + col];
            }
        }
        for (int ia = 0; ia < nci; ia++) {
            int ax = cart_lxyz[a0 + ia][0], ay = cart_lxyz[a0 + ia][1], az = cart_lxyz[a0 + ia][2];
            double fa = cb * cart_fac[a0 + ia];
            for (int ib = 0; ib < ncj; ib++) {
                int bx = cart_lxyz[b0 + ib][0], by = cart_lxyz[b0 + ib][1], bz = cart_lxyz[b0 + ib][2];
                double f = fa * cart_fac[b0 + ib];
                int ab = ia * ncj + ib;
                const double *grow = nbc == 1 ? G + ab * gs : s->Gb + ab * mr;
                int tx = ax + bx, ty = ay + by, tz = az + bz;
                for (int t = 0; t < tx + 2; t++) {
                    double ex = PE(pr, bp, 0, ax, bx, t);
                    double dax = 2.0 * a * PE(pr, bp, 0, ax + 1, bx, t), dbx = 2.0 * b * PE(pr, bp, 0, ax, bx + 1, t);
                    if (ax > 0) dax -= ax * PE(pr, bp, 0, ax - 1, bx, t);
                    if (bx > 0) dbx -= bx * PE(pr, bp, 0, ax, bx - 1, t);
                    for (int u = 0; u < ty + 2; u++) {
                        if (t > tx && u > ty) break;
                        double ey = PE(pr, bp, 1, ay, by, u);
                        double day = 2.0 * a * PE(pr, bp, 1, ay + 1, by, u), dby = 2.0 * b * PE(pr, bp, 1, ay, by + 1, u);
                        if (ay > 0) day -= ay * PE(pr, bp, 1, ay - 1, by, u);
                        if (by > 0) dby -= by * PE(pr, bp, 1, ay, by - 1, u);
                        int vmax = (t <= tx && u <= ty) ? tz + 2 : tz + 1;
                        for (int v = 0; v < vmax; v++) {
                            int h = herm_idx[t][u][v];
                            double yv = 0.0;
                            for (int c = 0; c < ncol; c++) yv += grow[c] * s->X[h * s->xc + c];
                            yv *= f;
                            if (yv == 0.0) continue;
                            double ez = PE(pr, bp, 2, az, bz, v);
                            double daz = 2.0 * a * PE(pr, bp, 2, az + 1, bz, v), dbz = 2.0 * b * PE(pr, bp, 2, az, bz + 1, v);
                            if (az > 0) daz -= az * PE(pr, bp, 2, az - 1, bz, v);
                            if (bz > 0) dbz -= bz * PE(pr, bp, 2, az, bz - 1, v);
                            out[0] += yv * dax * ey * ez; out[1] += yv * ex * day * ez; out[2] += yv * ex * ey * daz;
                            out[3] += yv * dbx * ey * ez; out[4] += yv * ex * dby * ez; out[5] += yv * ex * ey * dbz;
                        }
                    }
                }
            }
        }
    }
}

/* integrals.py:1247-1369 (_eri_grad_kernel) + :1498-1520 (two_electron_gradient) */
void orc_grad2e_strided(PAIR_ARGS, const double *Q, double threshold, i64 nao, i64 natm, const double *Dc, i64 nx,
                        const double *Dx, double kfac, double *grad, i64 stride, i64 offset);

void orc_grad2e(PAIR_ARGS, const double *Q, double threshold, i64 nao, i64 natm, const double *Dc, i64 nx,
                const double *Dx, double kfac, double *grad) {
    orc_grad2e_strided(PAIR_PASS, Q, threshold, nao, natm, Dc, nx, Dx, kfac, grad, 1, 0);
}

/* bra pairs pb with pb % stride == offset only (stride 1: the whole gradient) */
void orc_grad2e_strided(PAIR_ARGS, const double *Q, double threshold, i64 nao, i64 natm, const double *Dc, i64 nx,
                        const double *Dx, double kfac, double *grad, i64 stride, i64 offset) {
    init_tables();
    Pairs pr = make_pairs(PAIR_PASS);
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    double *parts = calloc((size_t)nthr * natm * 3, sizeof(double));
    i64 mr = pr.maxrow;
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *g = parts + (size_t)tid * natm * 3;
        Scratch s = scratch_new(&pr, 1);
        double *G = malloc(sizeof(double) * mr * mr), *Gt = malloc(sizeof(double) * mr * mr);
        double gab[6], gcd[6];
#pragma omp for schedule(dynamic, 1)
        for (i64 pb = offset; pb < pr.npair; pb += stride) {
            i64 si = pr.pair_blocks[2 * pb], sj = pr.pair_blocks[2 * pb + 1];
            i64 aA = pr.blk_atom[si], aB = pr.blk_atom[sj];
            for (i64 pk = 0; pk <= pb; pk++) {
                i64 sk = pr.pair_blocks[2 * pk], sl = pr.pair_blocks[2 * pk + 1];
                i64 aC = pr.blk_atom[sk], aD = pr.blk_atom[sl];
                if (aA == aB && aB == aC && aC == aD) continue;
                if (Q[pb] * Q[pk] == 0.0) continue;
                int nab, nbc, ncd, nkc;
                pair_dims(&pr, pb, &nab, &nbc);
                pair_dims(&pr, pk, &ncd, &nkc);
                int nrow = nab * nbc, ncol = ncd * nkc;
                double deg = 0.5 * (si != sj ? 2.0 : 1.0) * (sk != sl ? 2.0 : 1.0) * (pb != pk ? 2.0 : 1.0);
                double gmax = 0.0;
                int nci = cart_off[pr.blk_l[si] + 1] - cart_off[pr.blk_l[si]];
                int ncj = cart_off[pr.blk_l[sj] + 1] - cart_off[pr.blk_l[sj]];
                int nck = cart_off[pr.blk_l[sk] + 1] - cart_off[pr.blk_l[sk]];
                int ncl = cart_off[pr.blk_l[sl] + 1] - cart_off[pr.blk_l[sl]];
                i64 nqj = pr.blk_ncon[sj], nql = pr.blk_ncon[sl];
                for (i64 qi = 0; qi < pr.blk_ncon[si]; qi++) for (int a = 0; a < nci; a++) {
                    i64 m = pr.blk_ao[si] + qi * nci + a;
                    for (i64 qj = 0; qj < nqj; qj++) for (int b = 0; b < ncj; b++) {
                        i64 n = pr.blk_ao[sj] + qj * ncj + b;
                        i64 r = (qi * nqj + qj) * nab + a * ncj + b;
                        for (i64 qk = 0; qk < pr.blk_ncon[sk]; qk++) for (int c = 0; c < nck; c++) {
                            i64 lam = pr.blk_ao[sk] + qk * nck + c;
                            for (i64 ql = 0; ql < nql; ql++) for (int d = 0; d < ncl; d++) {
                                i64 sg = pr.blk_ao[sl] + ql * ncl + d;
                                i64 cc = (qk * nql + ql) * ncd + c * ncl + d;
                                double v = Dc[m * nao + n] * Dc[lam * nao + sg];
                                for (i64 x = 0; x < nx; x++) {
                                    const double *X = Dx + x * nao * nao;
                                    v -= 0.5 * kfac * (X[m * nao + lam] * X[n * nao + sg] + X[m * nao + sg] * X[n * nao + lam]);
                                }
                                v *= deg;
                                G[r * mr + cc] = v; Gt[cc * mr + r] = v;
                                gmax = fmax(gmax, fabs(v));
                            }
                        }
                    }
                }
                if (Q[pb] * Q[pk] * gmax < threshold) continue;
                int need_bra = aA != aB, need_ket = aC != aD;
                if (!need_bra && !need_ket) {
                    if (nrow >= ncol) {
                        grad_pass(&pr, pb, pk, G, mr, &s, gab);
                        for (int d = 0; d < 3; d++) { double t = gab[d] + gab[3 + d]; g[aA * 3 + d] += t; g[aC * 3 + d] -= t; }
                    } else {
                        grad_pass(&pr, pk, pb, Gt, mr, &s, gcd);
                        for (int d = 0; d < 3; d++) { double t = gcd[d] + gcd[3 + d]; g[aC * 3 + d] += t; g[aA * 3 + d] -= t; }
                    }
                    continue;
                }
                if (need_bra) grad_pass(&pr, pb, pk, G, mr, &s, gab);
                if (need_ket) grad_pass(&pr, pk, pb, Gt, mr, &s, gcd);
                for (int d = 0; d < 3; d++) {
                    if (need_bra && need_ket) {
                        g[aA * 3 + d] += gab[d]; g[aB * 3 + d] += gab[3 + d];
                        g[aC * 3 + d] += gcd[d]; g[aD * 3 + d] += gcd[3 + d];
                    } else if (need_bra) {
                        g[aA * 3 + d] += gab[d]; g[aB * 3 + d] += gab[3 + d]; g[aC * 3 + d] -= gab[d] + gab[3 + d];
                    } else {
                        g[aC * 3 + d] += gcd[d]; g[aD * 3 + d] += gcd[3 + d]; g[aA * 3 + d] -= gcd[d] + gcd[3 + d];
                    }
                }
            }
        }
        free(G); free(Gt);
        scratch_free(&s);
    }
    for (i64 i = 0; i < natm * 3; i++) {
        double t = 0.0;
        for (int k = 0; k < nthr; k++) t += parts[(size_t)k * natm * 3 + i];
        grad[i] = t;
    }
    free(parts);
}

/* ===================================================== one-electron */

#define SHELL_ARGS i64 ns, const i64 *shell_atom, const i64 *shell_l, const i64 *shell_prim, \
    const i64 *shell_ao, const double *prim_exp, const double *prim_coef, const double *pos
#define E1(dd, i, j, t) E[(((dd) * 8 + (i)) * 8 + (j)) * 16 + (t)]

/* integrals.py:143-151 (_kin1d) on an E table of stride 8 x 16 */
static double kin1d(const double *Ed, int i, int j, double b) {
    double v = -2.0 * b * (2 * j + 1) * Ed[(i * 8 + j) * 16] + 4.0 * b * b * Ed[(i * 8 + j + 2) * 16];
    if (j >= 2) v += j * (j - 1) * Ed[(i * 8 + j - 2) * 16];
    return -0.5 * v;
}

/* integrals.py:154-221 (_overlap_type_kernel): S, T and r - O; nao x nao each, M is 3 x nao x nao */
void orc_overlap_type(SHELL_ARGS, i64 nao, const double *origin, double *S, double *T, double *M) {
    init_tables();
    double E[3 * 8 * 8 * 16];
    double sq_pi = sqrt(PI);
    for (i64 si = 0; si < ns; si++) {
        int li = (int)shell_l[si]; i64 ai = shell_atom[si], oi = shell_ao[si];
        int ci0 = cart_off[li], nci = cart_off[li + 1] - ci0;
        for (i64 sj = 0; sj <= si; sj++) {
            int lj = (int)shell_l[sj]; i64 aj = shell_atom[sj], oj = shell_ao[sj];
            int cj0 = cart_off[lj], ncj = cart_off[lj + 1] - cj0;
            for (i64 ka = shell_prim[si]; ka < shell_prim[si + 1]; ka++) {
                double a = prim_exp[ka];
                for (i64 kb = shell_prim[sj]; kb < shell_prim[sj + 1]; kb++) {
                    double b = prim_exp[kb], p = a + b, mu = a * b / p, sq = sq_pi / sqrt(p);
                    for (int d = 0; d < 3; d++) {
                        double xab = pos[3 * ai + d] - pos[3 * aj + d];
                        double e00 = exp(-mu * xab * xab) * sq;
                        if (d == 0) e00 *= prim_coef[ka] * prim_coef[kb];
                        hermite_e(li, lj + 2, a, b, xab, e00, E + d * 8 * 8 * 16, 8, 16);
                    }
                    double P[3];
                    for (int d = 0; d < 3; d++) P[d] = (a * pos[3 * ai + d] + b * pos[3 * aj + d]) / p - origin[d];
                    for (int ia = 0; ia < nci; ia++) {
                        int ix = cart_lxyz[ci0 + ia][0], iy = cart_lxyz[ci0 + ia][1], iz = cart_lxyz[ci0 + ia][2];
                        double fa = cart_fac[ci0 + ia];
                        for (int ib = 0; ib < ncj; ib++) {
                            int jx = cart_lxyz[cj0 + ib][0], jy = cart_lxyz[cj0 + ib][1], jz = cart_lxyz[cj0 + ib][2];
                            double f = fa * cart_fac[cj0 + ib];
                            double sx = E1(0, ix, jx, 0), sy = E1(1, iy, jy, 0), sz = E1(2, iz, jz, 0);
                            double kx = kin1d(E, ix, jx, b), ky = kin1d(E + 8 * 8 * 16, iy, jy, b);
                            double kz = kin1d(E + 2 * 8 * 8 * 16, iz, jz, b);
                            i64 m = oi + ia, n = oj + ib;
                            S[m * nao + n] += f * sx * sy * sz;
                            T[m * nao + n] += f * (kx * sy * sz + sx * ky * sz + sx * sy * kz);
                            M[0 * nao * nao + m * nao + n] += f * (E1(0, ix, jx, 1) + P[0] * sx) * sy * sz;
                            M[1 * nao * nao + m * nao + n] += f * sx * (E1(1, iy, jy, 1) + P[1] * sy) * sz;
                            M[2 * nao * nao + m * nao + n] += f * sx * sy * (E1(2, iz, jz, 1) + P[2] * sz);
                        }
                    }
                }
            }
            if (si != sj)
                for (i64 m = oi; m < oi + nci; m++)
                    for (i64 n = oj; n < oj + ncj; n++) {
                        S[n * nao + m] = S[m * nao + n]; T[n * nao + m] = T[m * nao + n];
                        for (int d = 0; d < 3; d++) M[d * nao * nao + n * nao + m] = M[d * nao * nao + m * nao + n];
                    }
        }
    }
}

static double herm3(const double *E, int ax, int ay, int az, int bx, int by, int bz, int h) {
    return E1(0, ax, bx, herm_tuv[h][0]) * E1(1, ay, by, herm_tuv[h][1]) * E1(2, az, bz, herm_tuv[h][2]);
}

static double dherm3_a(const double *E, int ax, int ay, int az, int bx, int by, int bz, int h, int d, double a) {
    int t = herm_tuv[h][0], u = herm_tuv[h][1], v = herm_tuv[h][2];
    double ex = E1(0, ax, bx, t), ey = E1(1, ay, by, u), ez = E1(2, az, bz, v);
    if (d == 0) { double dx = 2.0 * a * E1(0, ax + 1, bx, t); if (ax > 0) dx -= ax * E1(0, ax - 1, bx, t); return dx * ey * ez; }
    if (d == 1) { double dy = 2.0 * a * E1(1, ay + 1, by, u); if (ay > 0) dy -= ay * E1(1, ay - 1, by, u); return ex * dy * ez; }
    double dz = 2.0 * a * E1(2, az + 1, bz, v); if (az > 0) dz -= az * E1(2, az - 1, bz, v); return ex * ey * dz;
}

/* integrals.py:259-329 (_nuclear_kernel): V += -sum_C q_C <m|1/r_C|n> */
void orc_nuclear(SHELL_ARGS, i64 nao, i64 nc, const double *charges, const double *cpos, double *V) {
    init_tables();
    double E[3 * 8 * 8 * 16], R[NHTOT], Rt[NHTOT], Rsum[NHTOT];
    for (i64 si = 0; si < ns; si++) {
        int li = (int)shell_l[si]; i64 ai = shell_atom[si], oi = shell_ao[si];
        int ci0 = cart_off[li], nci = cart_off[li + 1] - ci0;
        for (i64 sj = 0; sj <= si; sj++) {
            int lj = (int)shell_l[sj]; i64 aj = shell_atom[sj], oj = shell_ao[sj];
            int cj0 = cart_off[lj], ncj = cart_off[lj + 1] - cj0;
            int L = li + lj, nhL = nh(L);
            for (i64 ka = shell_prim[si]; ka < shell_prim[si + 1]; ka++) {
                double a = prim_exp[ka];
                for (i64 kb = shell_prim[sj]; kb < shell_prim[sj + 1]; kb++) {
                    double b = prim_exp[kb], p = a + b, mu = a * b / p;
                    for (int d = 0; d < 3; d++) {
                        double xab = pos[3 * ai + d] - pos[3 * aj + d];
                        double e00 = exp(-mu * xab * xab);
                        if (d == 0) e00 *= prim_coef[ka] * prim_coef[kb];
                        hermite_e(li, lj, a, b, xab, e00, E + d * 8 * 8 * 16, 8, 16);
                    }
                    double bp = b / p;
                    for (int h = 0; h < nhL; h++) Rsum[h] = 0.0;
                    for (i64 c = 0; c < nc; c++) {
                        double X = (pos[3 * ai] - cpos[3 * c]) - bp * (pos[3 * ai] - pos[3 * aj]);
                        double Y = (pos[3 * ai + 1] - cpos[3 * c + 1]) - bp * (pos[3 * ai + 1] - pos[3 * aj + 1]);
                        double Z = (pos[3 * ai + 2] - cpos[3 * c + 2]) - bp * (pos[3 * ai + 2] - pos[3 * aj + 2]);
                        hermite_r(L, p, X, Y, Z, R, Rt);
                        double w = -charges[c] * 2.0 * PI / p;
                        for (int h = 0; h < nhL; h++) Rsum[h] += w * R[h];
                    }
                    for (int ia = 0; ia < nci; ia++) {
                        int ix = cart_lxyz[ci0 + ia][0], iy = cart_lxyz[ci0 + ia][1], iz = cart_lxyz[ci0 + ia][2];
                        double fa = cart_fac[ci0 + ia];
                        for (int ib = 0; ib < ncj; ib++) {
                            int jx = cart_lxyz[cj0 + ib][0], jy = cart_lxyz[cj0 + ib][1], jz = cart_lxyz[cj0 + ib][2];
                            double acc = 0.0;
                            for (int h = 0; h < nhL; h++) acc += herm3(E, ix, iy, iz, jx, jy, jz, h) * Rsum[h];
                            V[(oi + ia) * nao + oj + ib] += fa * cart_fac[cj0 + ib] * acc;
                        }
                    }
                }
            }
            if (si != sj)
                for (i64 m = oi; m < oi + nci; m++)
                    for (i64 n = oj; n < oj + ncj; n++) V[n * nao + m] = V[m * nao + n];
        }
    }
}

/* integrals.py:332-404 (_overlap_kinetic_grad_kernel): grad += d/dR [sum W S + sum D T] */
void orc_ovlp_kin_grad(SHELL_ARGS, i64 nao, const double *W, const double *D, double *grad) {
    init_tables();
    double E[3 * 8 * 8 * 16], sq_pi = sqrt(PI);
    for (i64 si = 0; si < ns; si++) {
        int li = (int)shell_l[si]; i64 ai = shell_atom[si], oi = shell_ao[si];
        int ci0 = cart_off[li], nci = cart_off[li + 1] - ci0;
        for (i64 sj = 0; sj < si; sj++) {
            i64 aj = shell_atom[sj];
            if (aj == ai) continue;
            int lj = (int)shell_l[sj]; i64 oj = shell_ao[sj];
            int cj0 = cart_off[lj], ncj = cart_off[lj + 1] - cj0;
            double g[3] = {0.0, 0.0, 0.0};
            for (i64 ka = shell_prim[si]; ka < shell_prim[si + 1]; ka++) {
                double a = prim_exp[ka];
                for (i64 kb = shell_prim[sj]; kb < shell_prim[sj + 1]; kb++) {
                    double b = prim_exp[kb], p = a + b, mu = a * b / p, sq = sq_pi / sqrt(p);
                    for (int d = 0; d < 3; d++) {
                        double xab = pos[3 * ai + d] - pos[3 * aj + d];
                        double e00 = exp(-mu * xab * xab) * sq;
                        if (d == 0) e00 *= prim_coef[ka] * prim_coef[kb];
                        hermite_e(li + 1, lj + 2, a, b, xab, e00, E + d * 8 * 8 * 16, 8, 16);
                    }
                    for (int ia = 0; ia < nci; ia++) {
                        double fa = cart_fac[ci0 + ia];
                        for (int ib = 0; ib < ncj; ib++) {
                            double f = 2.0 * fa * cart_fac[cj0 + ib];
                            double wmn = f * W[(oi + ia) * nao + oj + ib], dmn = f * D[(oi + ia) * nao + oj + ib];
                            double S1[3], K1[3], dS[3], dK[3];
                            for (int d = 0; d < 3; d++) {
                                const double *Ed = E + d * 8 * 8 * 16;
                                int i = cart_lxyz[ci0 + ia][d], j = cart_lxyz[cj0 + ib][d];
                                S1[d] = Ed[(i * 8 + j) * 16];
                                K1[d] = kin1d(Ed, i, j, b);
                                dS[d] = 2.0 * a * Ed[((i + 1) * 8 + j) * 16];
                                dK[d] = 2.0 * a * kin1d(Ed, i + 1, j, b);
                                if (i > 0) { dS[d] -= i * Ed[((i - 1) * 8 + j) * 16]; dK[d] -= i * kin1d(Ed, i - 1, j, b); }
                            }
                            g[0] += wmn * dS[0] * S1[1] * S1[2] + dmn * (dK[0] * S1[1] * S1[2] + dS[0] * (K1[1] * S1[2] + S1[1] * K1[2]));
                            g[1] += wmn * S1[0] * dS[1] * S1[2] + dmn * (dK[1] * S1[0] * S1[2] + dS[1] * (K1[0] * S1[2] + S1[0] * K1[2]));
                            g[2] += wmn * S1[0] * S1[1] * dS[2] + dmn * (dK[2] * S1[0] * S1[1] + dS[2] * (K1[0] * S1[1] + S1[0] * K1[1]));
                        }
                    }
                }
            }
            for (int d = 0; d < 3; d++) { grad[ai * 3 + d] += g[d]; grad[aj * 3 + d] -= g[d]; }
        }
    }
}

/* integrals.py:407-501 (_nuclear_grad_kernel): grad += d/dR sum D V (basis and operator centres) */
void orc_nuclear_grad(SHELL_ARGS, i64 nao, i64 natm, const double *charges, const double *D, double *grad) {
    init_tables();
    double E[3 * 8 * 8 * 16], R[NHTOT], Rt[NHTOT], dE[NHTOT], dA[3][NHTOT];
    for (i64 si = 0; si < ns; si++) {
        int li = (int)shell_l[si]; i64 ai = shell_atom[si], oi = shell_ao[si];
        int ci0 = cart_off[li], nci = cart_off[li + 1] - ci0;
        for (i64 sj = 0; sj <= si; sj++) {
            int lj = (int)shell_l[sj]; i64 aj = shell_atom[sj], oj = shell_ao[sj];
            int cj0 = cart_off[lj], ncj = cart_off[lj + 1] - cj0;
            int L = li + lj, nhL = nh(L), nh1 = nh(L + 1);
            double sym = si != sj ? 2.0 : 1.0;
            for (i64 ka = shell_prim[si]; ka < shell_prim[si + 1]; ka++) {
                double a = prim_exp[ka];
                for (i64 kb = shell_prim[sj]; kb < shell_prim[sj + 1]; kb++) {
                    double b = prim_exp[kb], p = a + b, mu = a * b / p;
                    for (int d = 0; d < 3; d++) {
                        double xab = pos[3 * ai + d] - pos[3 * aj + d];
                        double e00 = exp(-mu * xab * xab);
                        if (d == 0) e00 *= prim_coef[ka] * prim_coef[kb];
                        hermite_e(li + 1, lj, a, b, xab, e00, E + d * 8 * 8 * 16, 8, 16);
                    }
                    for (int h = 0; h < nh1; h++) { dE[h] = 0.0; dA[0][h] = dA[1][h] = dA[2][h] = 0.0; }
                    for (int ia = 0; ia < nci; ia++) {
                        int ix = cart_lxyz[ci0 + ia][0], iy = cart_lxyz[ci0 + ia][1], iz = cart_lxyz[ci0 + ia][2];
                        double fa = cart_fac[ci0 + ia];
                        for (int ib = 0; ib < ncj; ib++) {
                            int jx = cart_lxyz[cj0 + ib][0], jy = cart_lxyz[cj0 + ib][1], jz = cart_lxyz[cj0 + ib][2];
                            double w = sym * fa * cart_fac[cj0 + ib] * D[(oi + ia) * nao + oj + ib];
                            if (w == 0.0) continue;
                            for (int h = 0; h < nhL; h++) dE[h] += w * herm3(E, ix, iy, iz, jx, jy, jz, h);
                            for (int h = 0; h < nh1; h++)
                                for (int d = 0; d < 3; d++) dA[d][h] += w * dherm3_a(E, ix, iy, iz, jx, jy, jz, h, d, a);
                        }
                    }
                    double bp = b / p;
                    for (i64 c = 0; c < natm; c++) {
                        double X = (pos[3 * ai] - pos[3 * c]) - bp * (pos[3 * ai] - pos[3 * aj]);
                        double Y = (pos[3 * ai + 1] - pos[3 * c + 1]) - bp * (pos[3 * ai + 1] - pos[3 * aj + 1]);
                        double Z = (pos[3 * ai + 2] - pos[3 * c + 2]) - bp * (pos[3 * ai + 2] - pos[3 * aj + 2]);
                        hermite_r(L + 1, p, X, Y, Z, R, Rt);
                        double pref = -charges[c] * 2.0 * PI / p;
                        for (int d = 0; d < 3; d++) {
                            double gA = 0.0, gC = 0.0;
                            for (int h = 0; h < nh1; h++) gA += dA[d][h] * R[h];
                            for (int h = 0; h < nhL; h++) {
                                int tuv[3] = {herm_tuv[h][0], herm_tuv[h][1], herm_tuv[h][2]};
                                tuv[d] += 1;
                                gC -= dE[h] * R[herm_idx[tuv[0]][tuv[1]][tuv[2]]];
                            }
                            gA *= pref; gC *= pref;
                            grad[ai * 3 + d] += gA; grad[c * 3 + d] += gC; grad[aj * 3 + d] -= gA + gC;
                        }
                    }
                }
            }
        }
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
