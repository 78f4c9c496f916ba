// Contracted block-quartet ERIs and their integral-direct J/K digestion.
//
// Work decomposition (one launch per bra pair class X):
//   * one CTA per bra block pair P1 (class X, in Schwarz-sorted order);
//   * the ket block pairs P2 of every class Y <= X that pass Q1 Q2 >= thr are
//     a prefix of class Y's Q-sorted list (cut at P1's own position for
//     Y == X, so each unordered pair of pairs is visited once);
//   * one thread item = (ket pair P2, ket Cartesian component pair cd): it
//     computes the column (ab|cd) for every bra row ab and every contraction
//     combination, by McMurchie-Davidson: per primitive quartet R_tuv up to
//     L = l_a+l_b+l_c+l_d, the ket Hermite->Cartesian step for its own cd,
//     and after the ket primitive loop the bra step (the reference's
//     _eri_block, aimd/qc/integrals.py:777-842, reorganised by column).
// The bra pair's primitive E tables are staged once per CTA in shared
// memory. Digestion: every exchange image of the 8-fold symmetry lands in a
// row of the bra pair's functions, so K rows are accumulated in shared
// memory and flushed once per CTA; J_ab accumulates in registers; only
// J_cd goes straight to global memory.
#pragma once
#include "hf_device.cuh"

namespace hf {

template <int CX, int CY>
struct QClass {
    static constexpr int LA = cls_la(CX), LB = cls_lb(CX), LC = cls_la(CY), LD = cls_lb(CY);
    static constexpr int LAB = LA + LB, LCD = LC + LD, L = LAB + LCD;
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND;
    static constexpr int KA = ncon_cap(LA), KB = ncon_cap(LB), KC = ncon_cap(LC), KD = ncon_cap(LD);
    static constexpr int KAB = KA * KB, KCD = KC * KD;
    static constexpr int NROW = KAB * NAB;
    // ket contraction combinations per thread item: all of them unless the
    // per-thread accumulator v[NROW][KG] would exceed 24 doubles
    static constexpr int KG = NROW * KCD <= 24 ? KCD : ((KCD % 2 == 0 && NROW * 2 <= 24) ? 2 : 1);
    static constexpr int NKG = KCD / KG;
    static constexpr int NHB = nherm(LAB);
    // R_tuv staged once per primitive quartet for all columns of a ket pair
    // (two-stage items): for dd bras against dp and dd kets, whose pairs have
    // one to three primitive pairs, 18-36 columns and L = 7-8, so that the
    // staged sub-chunks hold many items (measured: staging the classes with
    // many-primitive pairs starved the sub-chunks and was slower)
    static constexpr bool RSMEM = CX == 5 && CY >= 4;
    // Column-blocked items: one item covers the NC columns (ic, id) of one
    // id, so R_tuv of a primitive quartet is computed once for NC columns
    // instead of once per column; for the s/p bra classes against p kets,
    // where the NC x NROW x KG accumulators fit in registers
    static constexpr bool CBLK = (CX == 1 || CX == 2) && CY >= 1;
    static constexpr int NCB = CBLK ? NC : 1;       // columns per item
    static constexpr int NITEM = NCD / NCB;         // column items per ket pair and contraction group
};

// Bra-side E tables with an extra +G in i and j (G = 1 for gradients).
template <int LA, int LB, int G>
struct BraE {
    static constexpr int I = LA + 1 + G, J = LB + 1 + G, T = LA + LB + 1 + 2 * G;
    static constexpr int SIZE = 3 * I * J * T;
    __device__ static int at(int d, int i, int j, int t) { return ((d * I + i) * J + j) * T + t; }
};

// Shared-memory stage of one bra pair. The E tables and per-primitive
// scalars are held in the arithmetic type RT of the kernel that reads them
// (double, or float for the mixed-precision quartets); they are computed in
// FP64 either way.
constexpr int SBW = 12;     // per bra primitive: p, 1/p, Px, Py, Pz, a, b, -, c0..c3
template <typename RT>
struct BraStageT {
    int P1, A, B, nbp, aA, aB;
    int nA, nB, oA, oB;
    const double* rec;      // bra primitive records (global)
    RT* E;                  // [nbp][BraE::SIZE] (shared)
    RT* SB;                 // [nbp][SBW] (shared)
    RT* D;                  // gradients: [nbp][BraD::SIZE] derivative coefficients (shared)
};
using BraStage = BraStageT<double>;

// Fill the shared stage (E tables and scalars) for all bra primitives.
template <int LA, int LB, int G, typename RT>
__device__ __forceinline__ void stage_bra_e(const BraStageT<RT>& st) {
    using BE = BraE<LA, LB, G>;
    for (int w = threadIdx.x; w < st.nbp * 3; w += blockDim.x) {
        const int ib = w / 3, d = w % 3;
        const double* b = st.rec + (size_t)ib * PPW;
        const double p = b[0] + b[1];
        double e[LA + 1 + G][LB + 1 + G][LA + LB + 1 + 2 * G];
        hermite_e<LA + G, LB + G>(b[6 + d], b[9 + d], 0.5 / p, d == 0 ? b[2] : 1.0, e);
        RT* out = st.E + (size_t)ib * BE::SIZE;
#pragma unroll
        for (int i = 0; i < LA + 1 + G; ++i)
#pragma unroll
            for (int j = 0; j < LB + 1 + G; ++j)
#pragma unroll
                for (int t = 0; t < LA + LB + 1 + 2 * G; ++t) out[BE::at(d, i, j, t)] = static_cast<RT>(e[i][j][t]);
    }
    for (int ib = threadIdx.x; ib < st.nbp; ib += blockDim.x) {
        const double* b = st.rec + (size_t)ib * PPW;
        RT* o = st.SB + (size_t)ib * SBW;
        const double p = b[0] + b[1];
        const double vals[SBW] = {p, 1.0 / p, b[3], b[4], b[5], b[0], b[1], 0.0, b[12], b[13], b[14], b[15]};
#pragma unroll
        for (int i = 0; i < SBW; ++i) o[i] = static_cast<RT>(vals[i]);
    }
}

// One primitive-pair record of a ket pair (16 doubles, 128-byte aligned),
// loaded with 16-byte vector loads, held in the kernel's arithmetic type.
template <typename RT>
struct KetRecT {
    RT a, b, K, Qx, Qy, Qz, QAx, QAy, QAz, QBx, QBy, QBz, c[4];
};
template <typename RT>
__device__ __forceinline__ KetRecT<RT> load_ket(const double* __restrict__ rec) {
    const double2* r2 = reinterpret_cast<const double2*>(rec);
    KetRecT<RT> k;
    double2 v = __ldg(r2 + 0); k.a = (RT)v.x; k.b = (RT)v.y;
    v = __ldg(r2 + 1); k.K = (RT)v.x; k.Qx = (RT)v.y;
    v = __ldg(r2 + 2); k.Qy = (RT)v.x; k.Qz = (RT)v.y;
    v = __ldg(r2 + 3); k.QAx = (RT)v.x; k.QAy = (RT)v.y;
    v = __ldg(r2 + 4); k.QAz = (RT)v.x; k.QBx = (RT)v.y;
    v = __ldg(r2 + 5); k.QBy = (RT)v.x; k.QBz = (RT)v.y;
    v = __ldg(r2 + 6); k.c[0] = (RT)v.x; k.c[1] = (RT)v.y;
    v = __ldg(r2 + 7); k.c[2] = (RT)v.x; k.c[3] = (RT)v.y;
    return k;
}

__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }

// out[t] = e[i][j][t] for runtime (i, j), by predicated copies (no local memory).
template <int IM, int JM, int T, typename RT>
__device__ __forceinline__ void select_row(const RT (&e)[IM + 1][JM + 1][T + 1], int i, int j, RT (&out)[T + 1]) {
#pragma unroll
    for (int t = 0; t <= T; ++t) out[t] = RT(0);
#pragma unroll
    for (int ii = 0; ii <= IM; ++ii)
#pragma unroll
        for (int jj = 0; jj <= JM; ++jj)
            if (ii == i && jj == j)
#pragma unroll
                for (int t = 0; t <= T; ++t) out[t] = e[ii][jj][t];
}

// out[i][t] = e[i][j][t] for every i (runtime j), by predicated copies.
template <int IM, int JM, int T, typename RT>
__device__ __forceinline__ void select_j(const RT (&e)[IM + 1][JM + 1][T + 1], int j, RT (&out)[IM + 1][T + 1]) {
#pragma unroll
    for (int i = 0; i <= IM; ++i)
#pragma unroll
        for (int t = 0; t <= T; ++t) {
            RT x = e[i][0][t];
#pragma unroll
            for (int jj = 1; jj <= JM; ++jj)
                if (jj == j) x = e[i][jj][t];
            out[i][t] = x;
        }
}

// v[r][kk] = (row r | cd, contraction kk) of the quartet (staged bra pair,
// ket pair records rk with nkp primitive pairs); r = (ka*nB + kb)*NAB +
// ia*NB + jb, kk = kc*nD + kd - kg*KG (compact contraction indices over the
// blocks' actual counts).
// Loop order: bra primitives outer; for each, the ket primitives inner,
// where the ket step X_tuv (bra Hermite index tuv) of every primitive
// quartet is summed with its ket contraction coefficients,
// Xs[kk]_tuv = sum_ik c_ik[kk] X_tuv(ib, ik); the bra Hermite->Cartesian
// step, linear in X, then runs once per bra primitive instead of once per
// primitive quartet (the reference applies it per primitive quartet,
// aimd/qc/integrals.py:777-842).
// RS = false: R_tuv of each primitive quartet is computed here; RS = true:
// it is read from Rs, [ik][ib][NH(L)] pref * R_tuv staged by the CTA
// (stage_r below) once for all the columns of the ket pair.
template <int CX, int CY, typename RT, bool RS = false>
__device__ __forceinline__ void eri_column_bra_outer(const BraStageT<RT>& st, const double* __restrict__ rk, int nkp, int ic,
                                           int id, int kg, RT (&v)[QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                           const RT* __restrict__ Rs, int ib0, int ib1) {
    using Q = QClass<CX, CY>;
    using BE = BraE<Q::LA, Q::LB, 0>;
    constexpr int LA = Q::LA, LB = Q::LB, LC = Q::LC, LD = Q::LD, LAB = Q::LAB, LCD = Q::LCD, L = Q::L;
    // classes with L >= 6 keep their outer Hermite loops rolled (compile time)
    constexpr int UH = L >= 6 ? 1 : 16;
    const int cx = cart_x(LC, ic), cy = cart_y(LC, ic), cz = cart_z(LC, ic);
    const int dx = cart_x(LD, id), dy = cart_y(LD, id), dz = cart_z(LD, id);
    const RT fcd = static_cast<RT>(cart_norm(cx, cy, cz) * cart_norm(dx, dy, dz));
#pragma unroll
    for (int r = 0; r < Q::NROW; ++r)
#pragma unroll
        for (int k = 0; k < Q::KG; ++k) v[r][k] = RT(0);
    for (int ib = ib0; ib < ib1; ++ib) {
        const RT* sb = st.SB + ib * SBW;
        RT Xs[Q::KG][Q::NHB];
#pragma unroll
        for (int k = 0; k < Q::KG; ++k)
#pragma unroll
            for (int h = 0; h < Q::NHB; ++h) Xs[k][h] = RT(0);
        for (int ik = 0; ik < nkp; ++ik) {
            const KetRecT<RT> k = load_ket<RT>(rk + (size_t)ik * PPW);
            const RT q = k.a + k.b, oo2q = RT(0.5) / q;
            // ket E coefficients of this column only (box t2 <= cx+dx, ...)
            RT ex[LCD + 1], ey[LCD + 1], ez[LCD + 1];
            {
                RT e[LC + 1][LD + 1][LCD + 1];
                hermite_e<LC, LD>(k.QAx, k.QBx, oo2q, k.K, e);
                select_row<LC, LD, LCD>(e, cx, dx, ex);
                hermite_e<LC, LD>(k.QAy, k.QBy, oo2q, RT(1), e);
                select_row<LC, LD, LCD>(e, cy, dy, ey);
                hermite_e<LC, LD>(k.QAz, k.QBz, oo2q, RT(1), e);
                select_row<LC, LD, LCD>(e, cz, dz, ez);
            }
            RT ck[Q::KG];
#pragma unroll
            for (int i = 0; i < Q::KG; ++i) {
                RT c = k.c[0];
#pragma unroll
                for (int j = 1; j < Q::KCD; ++j)
                    if (j == kg * Q::KG + i) c = k.c[j];
                ck[i] = c * fcd;
            }
            // ket step: Xs[kk]_tuv += ck[kk] pref sum_{box(cd)} (-1)^|k| E^{cd}_k R_{tuv+k}
            auto ket_step = [&](const auto& R, RT scale) {
                RT sc[Q::KG];
#pragma unroll
                for (int kk = 0; kk < Q::KG; ++kk) sc[kk] = scale * ck[kk];
#pragma unroll UH
                for (int t = 0; t <= LAB; ++t)
#pragma unroll UH
                    for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
                        for (int w = 0; w <= LAB - t - u; ++w) {
                            RT s = RT(0);
#pragma unroll
                            for (int t2 = 0; t2 <= LCD; ++t2) {
                                if (t2 > cx + dx) continue;
#pragma unroll
                                for (int u2 = 0; u2 <= LCD; ++u2) {
                                    if (u2 > cy + dy) continue;
                                    const RT exy = ((t2 + u2) & 1) ? -ex[t2] * ey[u2] : ex[t2] * ey[u2];
#pragma unroll
                                    for (int v2 = 0; v2 <= LCD; ++v2) {
                                        if (v2 > cz + dz) continue;
                                        const RT e = (v2 & 1) ? -exy * ez[v2] : exy * ez[v2];
                                        s += e * R[hidx(t + t2, u + u2, w + v2)];
                                    }
                                }
                            }
#pragma unroll
                            for (int kk = 0; kk < Q::KG; ++kk) Xs[kk][hidx(t, u, w)] += sc[kk] * s;
                        }
            };
            if constexpr (RS) {
                ket_step(Rs + (size_t)(ik * st.nbp + ib) * nherm(L), RT(1));
            } else {
                const RT p = sb[0];
                const RT rs = rsqrt_t(p + q);
                const RT alpha = p * q * rs * rs;
                const RT pref = RT(TWO_PI_2_5) * sb[1] * (RT(2) * oo2q) * rs;
                RT R[nherm(L)];
                hermite_r<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, R);
                ket_step(R, pref);
            }
        }
        // bra step, once per bra primitive:
        // v[(ka,kb),ab][kk] += C[ka,kb] f_ab sum_box E^{ab}_tuv Xs[kk]_tuv
        const RT* E = st.E + (size_t)ib * BE::SIZE;
#pragma unroll UH
        for (int ia = 0; ia < Q::NA; ++ia) {
            const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
#pragma unroll
            for (int jb = 0; jb < Q::NB; ++jb) {
                const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                const RT fab = static_cast<RT>(cart_norm(ax, ay, az) * cart_norm(bx, by, bz));
                RT s[Q::KG];
#pragma unroll
                for (int kk = 0; kk < Q::KG; ++kk) s[kk] = RT(0);
#pragma unroll
                for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
                    for (int u = 0; u <= ay + by; ++u) {
                        const RT exy = E[BE::at(0, ax, bx, t)] * E[BE::at(1, ay, by, u)];
#pragma unroll
                        for (int w = 0; w <= az + bz; ++w) {
                            const RT e = exy * E[BE::at(2, az, bz, w)];
#pragma unroll
                            for (int kk = 0; kk < Q::KG; ++kk) s[kk] += e * Xs[kk][hidx(t, u, w)];
                        }
                    }
#pragma unroll
                for (int kab = 0; kab < Q::KAB; ++kab) {
                    const RT c = sb[8 + kab] * fab;
#pragma unroll
                    for (int kk = 0; kk < Q::KG; ++kk) v[kab * Q::NAB + ia * Q::NB + jb][kk] += c * s[kk];
                }
            }
        }
    }
}

// Ket primitives outermost, bra primitives inner, R_tuv and the bra step per
// primitive quartet: the order for bra pairs with many primitives (ss, ps,
// pp), where repeating the ket setup per bra primitive would cost more than
// the bra steps it saves.
template <int CX, int CY, typename RT>
__device__ __forceinline__ void eri_column_ket_outer(const BraStageT<RT>& st, const double* __restrict__ rk, int nkp,
                                                     int ic, int id, int kg, RT (&v)[QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                                     int ib0, int ib1) {
    using Q = QClass<CX, CY>;
    using BE = BraE<Q::LA, Q::LB, 0>;
    constexpr int LA = Q::LA, LB = Q::LB, LC = Q::LC, LD = Q::LD, LAB = Q::LAB, LCD = Q::LCD, L = Q::L;
    // classes with L >= 6 keep their outer Hermite loops rolled (compile time)
    constexpr int UH = L >= 6 ? 1 : 16;
    const int cx = cart_x(LC, ic), cy = cart_y(LC, ic), cz = cart_z(LC, ic);
    const int dx = cart_x(LD, id), dy = cart_y(LD, id), dz = cart_z(LD, id);
    const RT fcd = static_cast<RT>(cart_norm(cx, cy, cz) * cart_norm(dx, dy, dz));
#pragma unroll
    for (int r = 0; r < Q::NROW; ++r)
#pragma unroll
        for (int k = 0; k < Q::KG; ++k) v[r][k] = RT(0);
    for (int ik = 0; ik < nkp; ++ik) {
        const KetRecT<RT> k = load_ket<RT>(rk + (size_t)ik * PPW);
        const RT q = k.a + k.b, oo2q = RT(0.5) / q, iq = RT(2) * oo2q;
        // ket E coefficients of this column only (box t2 <= cx+dx, ...)
        RT ex[LCD + 1], ey[LCD + 1], ez[LCD + 1];
        {
            RT e[LC + 1][LD + 1][LCD + 1];
            hermite_e<LC, LD>(k.QAx, k.QBx, oo2q, k.K, e);
            select_row<LC, LD, LCD>(e, cx, dx, ex);
            hermite_e<LC, LD>(k.QAy, k.QBy, oo2q, RT(1), e);
            select_row<LC, LD, LCD>(e, cy, dy, ey);
            hermite_e<LC, LD>(k.QAz, k.QBz, oo2q, RT(1), e);
            select_row<LC, LD, LCD>(e, cz, dz, ez);
        }
        RT ck[Q::KG];
#pragma unroll
        for (int i = 0; i < Q::KG; ++i) {
            RT c = k.c[0];
#pragma unroll
            for (int j = 1; j < Q::KCD; ++j)
                if (j == kg * Q::KG + i) c = k.c[j];
            ck[i] = c * fcd;
        }
        for (int ib = ib0; ib < ib1; ++ib) {
            const RT* sb = st.SB + ib * SBW;
            const RT p = sb[0];
            const RT rs = rsqrt_t(p + q);
            const RT alpha = p * q * rs * rs;
            const RT pref = RT(TWO_PI_2_5) * sb[1] * iq * rs;
            RT R[nherm(L)];
            hermite_r<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, R);
            RT X[Q::NHB];
#pragma unroll UH
            for (int t = 0; t <= LAB; ++t)
#pragma unroll UH
                for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
                    for (int w = 0; w <= LAB - t - u; ++w) {
                        RT s = RT(0);
#pragma unroll
                        for (int t2 = 0; t2 <= LCD; ++t2) {
                            if (t2 > cx + dx) continue;
#pragma unroll
                            for (int u2 = 0; u2 <= LCD; ++u2) {
                                if (u2 > cy + dy) continue;
                                const RT exy = ((t2 + u2) & 1) ? -ex[t2] * ey[u2] : ex[t2] * ey[u2];
#pragma unroll
                                for (int v2 = 0; v2 <= LCD; ++v2) {
                                    if (v2 > cz + dz) continue;
                                    const RT e = (v2 & 1) ? -exy * ez[v2] : exy * ez[v2];
                                    s += e * R[hidx(t + t2, u + u2, w + v2)];
                                }
                            }
                        }
                        X[hidx(t, u, w)] = pref * s;
                    }
            // bra step: v[(ka,kb),ab][kk] += C[ka,kb] f_ab sum_box E^{ab}_tuv X[tuv] ck[kk]
            const RT* E = st.E + (size_t)ib * BE::SIZE;
#pragma unroll UH
            for (int ia = 0; ia < Q::NA; ++ia) {
                const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
#pragma unroll
                for (int jb = 0; jb < Q::NB; ++jb) {
                    const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                    const RT fab = static_cast<RT>(cart_norm(ax, ay, az) * cart_norm(bx, by, bz));
                    RT s = RT(0);
#pragma unroll
                    for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
                        for (int u = 0; u <= ay + by; ++u) {
                            const RT exy = E[BE::at(0, ax, bx, t)] * E[BE::at(1, ay, by, u)];
#pragma unroll
                            for (int w = 0; w <= az + bz; ++w) s += exy * E[BE::at(2, az, bz, w)] * X[hidx(t, u, w)];
                        }
                    s *= fab;
#pragma unroll
                    for (int kab = 0; kab < Q::KAB; ++kab) {
                        const RT c = sb[8 + kab] * s;
#pragma unroll
                        for (int kk = 0; kk < Q::KG; ++kk) v[kab * Q::NAB + ia * Q::NB + jb][kk] += c * ck[kk];
                    }
                }
            }
        }
    }
}

// v[ic][r][kk] = (row r | ic id, contraction kk) for the NC columns of one
// id (column-blocked items): the ket-outer order with R_tuv of each
// primitive quartet computed once and applied to every column; the ket E
// rows of a column come from the per-primitive table at compile-time ic.
template <int CX, int CY, typename RT>
__device__ __forceinline__ void eri_cols_ket_outer(const BraStageT<RT>& st, const double* __restrict__ rk, int nkp,
                                                   int id, int kg,
                                                   RT (&v)[QClass<CX, CY>::NC][QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                                   int ib0, int ib1) {
    using Q = QClass<CX, CY>;
    using BE = BraE<Q::LA, Q::LB, 0>;
    constexpr int LA = Q::LA, LB = Q::LB, LC = Q::LC, LD = Q::LD, LAB = Q::LAB, LCD = Q::LCD, L = Q::L;
    const int dx = cart_x(LD, id), dy = cart_y(LD, id), dz = cart_z(LD, id);
    const RT fd = static_cast<RT>(cart_norm(dx, dy, dz));
#pragma unroll
    for (int c = 0; c < Q::NC; ++c)
#pragma unroll
        for (int r = 0; r < Q::NROW; ++r)
#pragma unroll
            for (int k = 0; k < Q::KG; ++k) v[c][r][k] = RT(0);
    for (int ik = 0; ik < nkp; ++ik) {
        const KetRecT<RT> k = load_ket<RT>(rk + (size_t)ik * PPW);
        const RT q = k.a + k.b, oo2q = RT(0.5) / q, iq = RT(2) * oo2q;
        // ket E of this id: ex[i][t] = E^{i, dx}_t for every i <= LC
        RT ex[LC + 1][LCD + 1], ey[LC + 1][LCD + 1], ez[LC + 1][LCD + 1];
        {
            RT e[LC + 1][LD + 1][LCD + 1];
            hermite_e<LC, LD>(k.QAx, k.QBx, oo2q, k.K, e);
            select_j<LC, LD, LCD>(e, dx, ex);
            hermite_e<LC, LD>(k.QAy, k.QBy, oo2q, RT(1), e);
            select_j<LC, LD, LCD>(e, dy, ey);
            hermite_e<LC, LD>(k.QAz, k.QBz, oo2q, RT(1), e);
            select_j<LC, LD, LCD>(e, dz, ez);
        }
        RT ck[Q::KG];
#pragma unroll
        for (int i = 0; i < Q::KG; ++i) {
            RT c = k.c[0];
#pragma unroll
            for (int j = 1; j < Q::KCD; ++j)
                if (j == kg * Q::KG + i) c = k.c[j];
            ck[i] = c * fd;
        }
        for (int ib = ib0; ib < ib1; ++ib) {
            const RT* sb = st.SB + ib * SBW;
            const RT p = sb[0];
            const RT rs = rsqrt_t(p + q);
            const RT alpha = p * q * rs * rs;
            const RT pref = RT(TWO_PI_2_5) * sb[1] * iq * rs;
            RT R[nherm(L)];
            hermite_r<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, R);
            const RT* E = st.E + (size_t)ib * BE::SIZE;
#pragma unroll
            for (int ic = 0; ic < Q::NC; ++ic) {
                const int cx = cart_x(LC, ic), cy = cart_y(LC, ic), cz = cart_z(LC, ic);
                const RT fc = static_cast<RT>(cart_norm(cx, cy, cz));
                RT X[Q::NHB];
#pragma unroll
                for (int t = 0; t <= LAB; ++t)
#pragma unroll
                    for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
                        for (int w = 0; w <= LAB - t - u; ++w) {
                            RT s = RT(0);
#pragma unroll
                            for (int t2 = 0; t2 <= LCD; ++t2) {
                                if (t2 > cx + dx) continue;
#pragma unroll
                                for (int u2 = 0; u2 <= LCD; ++u2) {
                                    if (u2 > cy + dy) continue;
                                    const RT exy = ((t2 + u2) & 1) ? -ex[cx][t2] * ey[cy][u2] : ex[cx][t2] * ey[cy][u2];
#pragma unroll
                                    for (int v2 = 0; v2 <= LCD; ++v2) {
                                        if (v2 > cz + dz) continue;
                                        const RT e = (v2 & 1) ? -exy * ez[cz][v2] : exy * ez[cz][v2];
                                        s += e * R[hidx(t + t2, u + u2, w + v2)];
                                    }
                                }
                            }
                            X[hidx(t, u, w)] = pref * fc * s;
                        }
                // bra step of column ic
#pragma unroll
                for (int ia = 0; ia < Q::NA; ++ia) {
                    const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
#pragma unroll
                    for (int jb = 0; jb < Q::NB; ++jb) {
                        const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                        const RT fab = static_cast<RT>(cart_norm(ax, ay, az) * cart_norm(bx, by, bz));
                        RT s = RT(0);
#pragma unroll
                        for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
                            for (int u = 0; u <= ay + by; ++u) {
                                const RT exy = E[BE::at(0, ax, bx, t)] * E[BE::at(1, ay, by, u)];
#pragma unroll
                                for (int w = 0; w <= az + bz; ++w) s += exy * E[BE::at(2, az, bz, w)] * X[hidx(t, u, w)];
                            }
                        s *= fab;
#pragma unroll
                        for (int kab = 0; kab < Q::KAB; ++kab) {
                            const RT c = sb[8 + kab] * s;
#pragma unroll
                            for (int kk = 0; kk < Q::KG; ++kk) v[ic][kab * Q::NAB + ia * Q::NB + jb][kk] += c * ck[kk];
                        }
                    }
                }
            }
        }
    }
}

// (row r | cd) of a quartet column: bra-outer order (the bra step once per
// bra primitive) for the d-shell bra classes, whose pairs have few
// primitives, and the ket-outer order for the others.
template <int CX, int CY, typename RT, bool RS = false>
__device__ __forceinline__ void eri_column(const BraStageT<RT>& st, const double* __restrict__ rk, int nkp, int ic,
                                           int id, int kg, RT (&v)[QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                           const RT* __restrict__ Rs, int ib0, int ib1) {
    if constexpr (RS || CX >= 3) eri_column_bra_outer<CX, CY, RT, RS>(st, rk, nkp, ic, id, kg, v, Rs, ib0, ib1);
    else eri_column_ket_outer<CX, CY, RT>(st, rk, nkp, ic, id, kg, v, ib0, ib1);
}

// Everything the quartet kernels share.
struct QuartetArgs {
    PairView pv;
    BlockView bv;
    const int* sorted;          // [npair] pair index at sorted position
    const double* sortedQ;      // [npair]
    const int64_t* counts;      // [NSEG][npair + 1] kept ket prefix length per (ket segment, bra position)
    // mixed precision: [NSEG][npair + 1] prefix with Q1 Q2 >= the FP32
    // cutoff (evaluated in FP64); the rest of the kept prefix runs in FP32.
    // nullptr: everything in FP64.
    const int64_t* counts_hi;
    const int* seg_start;       // [NSEG + 1] sorted position of each segment (device)
    int npair;
    int cls_start[NCLS + 1];    // sorted positions of each angular class (geometry independent)
    int nao;
};

// Ket range [b, e) of segment seg for bra position spos that the kernels of
// arithmetic type RT evaluate: the FP64 prefix, or the FP32 tail.
template <typename RT>
__device__ __forceinline__ void ket_range(const QuartetArgs& a, int seg, int spos, int64_t& b, int64_t& e) {
    const size_t i = (size_t)seg * (a.npair + 1) + spos;
    const int64_t cnt = a.counts[i];
    int64_t hi = cnt;
    if (a.counts_hi) hi = a.counts_hi[i] < cnt ? a.counts_hi[i] : cnt;
    if constexpr (sizeof(RT) == sizeof(double)) {
        b = 0;
        e = hi;
    } else {
        b = hi;
        e = a.counts_hi ? cnt : hi;
    }
}

// A thread's R_tuv in shared memory: element i at p[i * NT] (NT = threads
// of the CTA, p = base + threadIdx.x), so that a warp's accesses to one
// element fall in distinct banks. Frees the registers (or the local
// memory) that a large R array takes through the contraction passes.
template <typename RT, int NT>
struct RColumn {
    RT* p;
    __device__ __forceinline__ RT& operator[](int i) const { return p[i * NT]; }
};

// ---------------------------------------------------------------- work plan
// The class kernels are persistent: their CTAs take chunks of (bra pair,
// ket window) from a device counter until the launch's plan is used up, so
// that the few heavy bras (many primitives, long ket lists) are spread over
// many CTAs instead of setting the kernel's duration. A plan holds, per bra
// of the class, the exclusive prefix of its chunk counts; chunk j of nch
// covers the bra's work units [W j / nch, W (j + 1) / nch) in ket segment
// order. Work of a ket pair of segment sub: bra primitive pairs x twice
// the segment's typical ket primitive pairs x the column items per pair.
struct WorkPlan {
    const int* off;     // [nbra + 1] chunk prefix over the bras of the class (off[nbra]: chunks)
    int* next;          // chunk counter of the launch (zeroed with the plan)
};

__host__ __device__ constexpr int ket_prims2(int ppb) {
    return ppb == 0 ? 2 : ppb == 1 ? 5 : ppb == 2 ? 11 : ppb == 3 ? 23 : ppb == 4 ? 47 : 80;
}

template <int CX, int CY>
__device__ __forceinline__ int64_t ket_work(int sub);

// Work units of bra position spos against ket class CY in the ket ranges
// that the kernels of type RT evaluate.
template <int CX, int CY, typename RT>
__device__ int64_t bra_work(const QuartetArgs& q, int spos) {
    int64_t w = 0;
    for (int sub = 0; sub < NSUB; ++sub) {
        int64_t kb, ke;
        ket_range<RT>(q, CY * NSUB + sub, spos, kb, ke);
        if (ke > kb) w += (ke - kb) * ket_work<CX, CY>(sub);
    }
    return w * q.pv.npp[q.sorted[spos]];
}

// Kets [k0, k1) of a segment of len kets, each of weight wk, whose work
// starts inside the window [w0, w1) (acc: work of the segments before).
__device__ __forceinline__ void window_kets(int64_t w0, int64_t w1, int64_t acc, int64_t wk, int64_t len,
                                            int64_t& k0, int64_t& k1) {
    auto first = [&](int64_t x) { return x <= 0 ? int64_t(0) : ((x + wk - 1) / wk < len ? (x + wk - 1) / wk : len); };
    k0 = first(w0 - acc);
    k1 = first(w1 - acc);
}

// Chunk j of nch of a bra of W work units: [W j / nch, W (j + 1) / nch),
// without forming W j.
__device__ __forceinline__ int64_t chunk_edge(int64_t W, int j, int nch) {
    const int64_t q = W / nch, r = W % nch;
    return q * j + (r * j) / nch;
}

// The next chunk of the launch for this CTA: thread 0 takes it from the
// counter and finds its bra (last b with off[b] <= c); all threads return
// the same (c, b) and c >= off[nbra] when the plan is used up.
__device__ __forceinline__ void next_chunk(const WorkPlan& plan, int nbra, int* sh, int& c, int& b) {
    if (threadIdx.x == 0) {
        const int cc = atomicAdd(plan.next, 1);
        int lo = 0, hi = nbra;                          // off[lo] <= cc < off[hi] while cc < total
        if (cc < plan.off[nbra]) {
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (plan.off[mid] <= cc) lo = mid;
                else hi = mid;
            }
        }
        sh[0] = cc;
        sh[1] = lo;
    }
    __syncthreads();
    c = sh[0];
    b = sh[1];
}

template <typename RT>
__device__ __forceinline__ void load_stage(const QuartetArgs& a, int P1, BraStageT<RT>& st, RT* E) {
    st.P1 = P1;
    st.A = a.pv.pa_blk[P1];
    st.B = a.pv.pb_blk[P1];
    st.nbp = a.pv.npp[P1];
    st.rec = a.pv.rec + a.pv.slot[P1] * PPW;
    st.aA = a.bv.atom[st.A];
    st.aB = a.bv.atom[st.B];
    st.nA = a.bv.ncon[st.A];
    st.nB = a.bv.ncon[st.B];
    st.oA = a.bv.ao[st.A];
    st.oB = a.bv.ao[st.B];
    st.SB = E;                                   // [nbp][SBW] scalars, then the E tables
    st.E = E + (size_t)st.nbp * SBW;
}

struct JKArgs {
    QuartetArgs q;
    const double* D;    // [nset][nao][nao], symmetric
    facc* J;            // un-symmetrised accumulators, same shape (fixed point, scale *fix)
    facc* K;
    const double* fix;  // device scalar: the fixed-point scale of J and K (jk_fix_for(max |D|))
    // density-weighted screening (difference densities): skip a quartet when
    // Q1 Q2 max|D| over its six density blocks < dthr; bmax = nullptr: off
    const double* bmax; // [nblock][nblock] max |D| per block pair (all sets)
    int nblock;
    double dthr;
    size_t rbuf;        // elements of the kernel's staged-R buffer (set per launch)
    // 1: the K rows of the bra functions accumulate in global memory (set per
    // launch when the per-CTA shared rows, NF x nao doubles, would not fit)
    int kglobal;
    WorkPlan plan;      // chunks of the launch (set per launch)
    int item_pq;        // primitive quartets per split column item (launch shape)
};

// Digest one column (fixed ket component pair cd, all ket contractions kk)
// of a quartet for NS densities. Each tensor element the block reaches is
// visited n_gen = (A==B ? 2:1)(C==D ? 2:1)(P1==P2 ? 2:1) times under the 8
// index maps, so each image carries g = 1/n_gen:
//   J[m,n] += 2g v D[l,s],  J[l,s] += 2g v D[m,n]
//   K[m,l] += g v D[n,s],   K[n,l] += g v D[m,s],  K[m,s] += g v D[n,l],  K[n,s] += g v D[m,l]
// (m in A, n in B, l in C, s in D); the host forms J + J^T and K + K^T.
// K rows m, n belong to the bra pair: Ksm[set][slot][col], slot < KA*NA for
// A's functions, then B's.
template <int CX, int CY, int NS, bool KGLOBAL, typename ST>
__device__ __forceinline__ void jk_digest_column(const JKArgs& a, const ST& st, int P2, int C, int Dd, int ic,
                                                 int id, int kg,
                                                 const double (&v)[QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                                 double* Jt, facc* Ksm) {
    using Q = QClass<CX, CY>;
    const BlockView& bv = a.q.bv;
    const int nC = bv.ncon[C], nD = bv.ncon[Dd], oC = bv.ao[C], oD = bv.ao[Dd];
    const double g = 1.0 / ((st.A == st.B ? 2.0 : 1.0) * (C == Dd ? 2.0 : 1.0) * (st.P1 == P2 ? 2.0 : 1.0));
    const int n = a.q.nao;
    const size_t nn = (size_t)n * n;
    const double fx = __ldg(a.fix);
    constexpr int NFA = Q::KA * Q::NA;      // A slots, then B slots
    constexpr int NF = NFA + Q::KB * Q::NB;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const double* __restrict__ D = a.D + s * nn;
        // K rows of the bra functions: shared accumulator, or the global K
        // itself (KGLOBAL, for bra classes whose rows would not fit)
        const bool kgl = KGLOBAL || a.kglobal;
        facc* Ks = kgl ? nullptr : Ksm + (size_t)s * NF * n;
        facc* Kg = a.K + s * nn;
#pragma unroll
        for (int kk = 0; kk < Q::KG; ++kk) {
                const int kq = kg * Q::KG + kk;
                if (kq >= nC * nD) continue;
                const int kc = kq / nD, kd = kq % nD;
                const int l = oC + kc * Q::NC + ic, sg = oD + kd * Q::ND + id;
                const double dls = __ldg(D + (size_t)l * n + sg);
                double jcd = 0.0;
#pragma unroll
                for (int ka = 0; ka < Q::KA; ++ka)
#pragma unroll
                    for (int kb = 0; kb < Q::KB; ++kb) {
                        if (ka >= st.nA || kb >= st.nB) continue;
#pragma unroll
                        for (int ia = 0; ia < Q::NA; ++ia)
#pragma unroll
                            for (int jb = 0; jb < Q::NB; ++jb) {
                                const int r = (ka * st.nB + kb) * Q::NAB + ia * Q::NB + jb;
                                const int m = st.oA + ka * Q::NA + ia, nb_ = st.oB + kb * Q::NB + jb;
                                jcd += v[r][kk] * __ldg(D + (size_t)m * n + nb_);
                                Jt[(s * Q::NROW + r) * blockDim.x + threadIdx.x] += 2.0 * g * v[r][kk] * dls;
                            }
                    }
                fadd(a.J + s * nn + (size_t)l * n + sg, 2.0 * g * jcd, fx);
                // K[m, l] and K[m, sg]: rows of A's functions
#pragma unroll
                for (int ka = 0; ka < Q::KA; ++ka)
#pragma unroll
                    for (int ia = 0; ia < Q::NA; ++ia) {
                        if (ka >= st.nA) continue;
                        double s1 = 0.0, s2 = 0.0;
#pragma unroll
                        for (int kb = 0; kb < Q::KB; ++kb)
#pragma unroll
                            for (int jb = 0; jb < Q::NB; ++jb) {
                                if (kb >= st.nB) continue;
                                const int r = (ka * st.nB + kb) * Q::NAB + ia * Q::NB + jb;
                                const size_t nb_ = st.oB + kb * Q::NB + jb;
                                s1 += v[r][kk] * __ldg(D + nb_ * n + sg);
                                s2 += v[r][kk] * __ldg(D + nb_ * n + l);
                            }
                        facc* row = kgl ? Kg + (size_t)(st.oA + ka * Q::NA + ia) * n
                                              : Ks + (size_t)(ka * Q::NA + ia) * n;
                        fadd(row + l, g * s1, fx);
                        fadd(row + sg, g * s2, fx);
                    }
                // K[n, l] and K[n, sg]: rows of B's functions
#pragma unroll
                for (int kb = 0; kb < Q::KB; ++kb)
#pragma unroll
                    for (int jb = 0; jb < Q::NB; ++jb) {
                        if (kb >= st.nB) continue;
                        double s1 = 0.0, s2 = 0.0;
#pragma unroll
                        for (int ka = 0; ka < Q::KA; ++ka)
#pragma unroll
                            for (int ia = 0; ia < Q::NA; ++ia) {
                                if (ka >= st.nA) continue;
                                const int r = (ka * st.nB + kb) * Q::NAB + ia * Q::NB + jb;
                                const size_t m = st.oA + ka * Q::NA + ia;
                                s1 += v[r][kk] * __ldg(D + m * n + sg);
                                s2 += v[r][kk] * __ldg(D + m * n + l);
                            }
                        facc* row = kgl ? Kg + (size_t)(st.oB + kb * Q::NB + jb) * n
                                              : Ks + (size_t)(NFA + kb * Q::NB + jb) * n;
                        fadd(row + l, g * s1, fx);
                        fadd(row + sg, g * s2, fx);
                    }
            }
    }
}

// Items of ket class CY for the staged bra pair.
// Work queue of one CTA: the ket pairs of a segment that pass a per-pair
// test are compacted into shared memory in chunks of KQ_CAP (warp ballots,
// warps in index order), then dealt to the threads as NPER items each,
// so that lanes only receive live work. Dealing starts where the previous
// chunk ended (rot), so ragged tails do not pile up on the low threads.
// Every thread of the CTA must call this with the same j0 and cnt.
constexpr int KQ_CAP = 256;

// Ket contraction groups of KG combinations that a segment's pairs need: its
// pairs carry 1, 2 or 4 contraction combinations (sub-class contraction
// bucket), stored first in the compact index, so groups past them are empty.
template <int KG, int NKG>
__device__ __forceinline__ int seg_groups(int sub) {
    const int cb = sub % NCONB;
    const int ncs = cb == 0 ? 1 : (cb == 1 ? 2 : 4);
    const int g = (ncs + KG - 1) / KG;
    return g < NKG ? g : NKG;
}
template <int CX, int CY>
__device__ __forceinline__ int64_t ket_work(int sub) {
    using Q = QClass<CX, CY>;
    return (int64_t)ket_prims2(sub / NCONB) * Q::NCD * seg_groups<Q::KG, Q::NKG>(sub);
}

// Bra-primitive splits of the column items of a ket segment: an item of a
// pair of many primitive quartets would run them all in one thread while
// the rest of the CTA waits at the next barrier, so such items are split
// over ranges of the bra primitives (about item_pq quartets each, a launch
// shape of the context, default ITEM_PQ; the partial columns are linear in
// the quartets and are digested one by one).
constexpr int ITEM_PQ = 32;
__device__ __forceinline__ int bra_splits(int nbp, int sub, int item_pq) {
    const int s = nbp * ket_prims2(sub / NCONB) / (2 * item_pq);
    return s < 1 ? 1 : (s > nbp ? nbp : s);
}

struct KetQueue {
    int pos[KQ_CAP];
    int wcnt[32];           // per-warp counts of one compaction step
    int n;
};

// Compact the positions p0 .. p0+m-1 that pass keep() into q.pos[0 .. q.n)
// in position order (per-warp ballots, warps in index order), so that the
// queue, the item dealing and every per-thread partial sum are the same on
// every run. store(slot, pos) records what the caller needs per entry.
template <typename Queue, typename Keep, typename Store>
__device__ __forceinline__ void compact(Queue& q, int p0, int m, Keep keep, Store store) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int n = 0;
    for (int i0 = 0; i0 < m; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool k = i < m && keep(p0 + i);
        const unsigned mask = __ballot_sync(0xffffffffu, k);
        if (lane == 0) q.wcnt[warp] = __popc(mask);
        __syncthreads();
        int before = n, total = 0;
        for (int w = 0; w < nwarps; ++w) {
            const int c = q.wcnt[w];
            if (w < warp) before += c;
            total += c;
        }
        if (k) store(before + __popc(mask & ((1u << lane) - 1u)), p0 + i);
        n += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) q.n = n;
    __syncthreads();
}

template <typename Queue, typename Keep, typename Work>
__device__ __forceinline__ void ket_items(int nper, int j0, int64_t cnt, Queue& q, int& rot, Keep keep, Work work) {
    for (int64_t base = 0; base < cnt; base += KQ_CAP) {
        const int m = static_cast<int>(cnt - base < KQ_CAP ? cnt - base : KQ_CAP);
        compact(q, j0 + static_cast<int>(base), m, keep, [&](int slot, int pos) { q.pos[slot] = pos; });
        const int items = q.n * nper;
        int it = static_cast<int>(threadIdx.x) - rot;
        if (it < 0) it += blockDim.x;
        // column-major: neighbouring lanes take the same ket column of
        // different ket pairs, so the column's box conditions are warp-uniform
        const int nq = q.n;
        for (; it < items; it += blockDim.x) work(q.pos[it % nq], it / nq);
        rot = (rot + items) % static_cast<int>(blockDim.x);
        __syncthreads();
    }
}

// ---- Two-stage items: R_tuv staged in shared memory
// A ket pair of class Y carries NCD Cartesian columns (x contraction
// groups), each one work item; R_tuv of a primitive quartet is the same for
// all of them. For the classes where recomputing it per item costs (RSmem
// below), each queue chunk is cut into sub-chunks whose primitive quartets
// fit RB_PQ slots of a shared buffer (plus the largest single ket pair),
// and per sub-chunk:
//   stage 1: one thread per primitive quartet (ket pair i, ket primitive ik,
//            bra primitive ib) writes pref * R_tuv into the buffer;
//   stage 2: the column items of the sub-chunk's ket pairs read it.
template <int L, typename RT>
struct RSmem {
    static constexpr int NH = nherm(L);
    // slots per sub-chunk: about 32 KB of R (FP64; 16 KB of FP32 R)
    static constexpr int RB_PQ = (4096 + NH - 1) / NH;
    // R level recursion in shared memory instead of registers from this L on
    // (it would hold NH(L) values in registers for the whole kernel)
    static constexpr bool INPLACE = L >= 6;
};
template <int L, typename RT>
__host__ __device__ constexpr size_t rsmem_bytes(int max_bra_prims, int max_ket_prims) {
    return sizeof(RT) * (size_t)nherm(L) * (RSmem<L, RT>::RB_PQ + (size_t)max_bra_prims * max_ket_prims);
}

struct KetQueueR {
    int pos[KQ_CAP];
    int wcnt[32];           // per-warp counts of one compaction step
    int pq[KQ_CAP + 1];     // exclusive prefix of primitive quartets over the chunk's entries
    int sc[KQ_CAP];         // sub-chunk of each entry
    int n;
};

// first index in [lo, hi) with a[i] >= key (a non-decreasing)
__device__ __forceinline__ int lower_bound_i(const int* a, int lo, int hi, int key) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// pref * R_tuv of primitive quartet (bra primitive ib of the stage, ket
// primitive record kr) into out[NH(L)] (shared memory).
template <int L, typename RT>
__device__ __forceinline__ void stage_r(const BraStageT<RT>& st, int ib, const double* __restrict__ kr, RT* out) {
    const double2* r2 = reinterpret_cast<const double2*>(kr);
    const double2 ab = __ldg(r2 + 0), kq = __ldg(r2 + 1), qyz = __ldg(r2 + 2);
    const RT* sb = st.SB + ib * SBW;
    const RT p = sb[0], q = static_cast<RT>(ab.x) + static_cast<RT>(ab.y);
    const RT rs = rsqrt_t(p + q);
    const RT alpha = p * q * rs * rs;
    const RT pref = RT(TWO_PI_2_5) * sb[1] * (RT(1) / q) * rs;
    const RT X = sb[2] - static_cast<RT>(kq.y), Y = sb[3] - static_cast<RT>(qyz.x), Z = sb[4] - static_cast<RT>(qyz.y);
    if constexpr (RSmem<L, RT>::INPLACE) {
        hermite_r_scaled<L>(alpha, X, Y, Z, pref, out);
    } else {
        RT R[nherm(L)];
        hermite_r_scaled<L>(alpha, X, Y, Z, pref, R);
#pragma unroll
        for (int h = 0; h < nherm(L); ++h) out[h] = R[h];
    }
}

// ket_items with R staged per sub-chunk; work(pos, r, Rs) receives the ket
// pair's staged R ([ik][ib][NH(L)]). Rbuf holds rsmem_bytes(...) bytes.
template <int L, typename RT, typename Keep, typename Work>
__device__ __forceinline__ void ket_items_r(int nper, int j0, int64_t cnt, KetQueueR& q, int& rot,
                                            const BraStageT<RT>& st, const QuartetArgs& qa, RT* Rbuf, Keep keep,
                                            Work work) {
    constexpr int NH = nherm(L);
    constexpr int B = RSmem<L, RT>::RB_PQ;
    const int lane = threadIdx.x & 31;
    const int nbp = st.nbp;
    for (int64_t base = 0; base < cnt; base += KQ_CAP) {
        const int m = static_cast<int>(cnt - base < KQ_CAP ? cnt - base : KQ_CAP);
        compact(q, j0 + static_cast<int>(base), m, keep, [&](int slot, int pos) {
            q.pos[slot] = pos;
            q.pq[slot] = qa.pv.npp[qa.sorted[pos]] * nbp;          // primitive quartets of the entry
        });
        const int ne = q.n;
        if (ne == 0) continue;                                      // uniform: q.n is shared
        // warp 0: exclusive prefix of the entries' primitive quartets and
        // their sub-chunks (an entry belongs to the sub-chunk of its last slot)
        if (threadIdx.x < 32) {
            constexpr int PER = KQ_CAP / 32;
            int c[PER], local = 0;
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const int i = lane * PER + k;
                c[k] = i < ne ? q.pq[i] : 0;
                local += c[k];
            }
            int incl = local;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += v;
            }
            __syncwarp();
            int run = incl - local;
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const int i = lane * PER + k;
                if (i < ne) {
                    q.pq[i] = run;
                    q.sc[i] = (run + (c[k] > 0 ? c[k] : 1) - 1) / B;
                    run += c[k];
                }
            }
            if (lane == 31) q.pq[ne] = incl;
        }
        __syncthreads();
        const int k0 = q.sc[0], k1 = q.sc[ne - 1];
        for (int kc = k0; kc <= k1; ++kc) {
            const int f = lower_bound_i(q.sc, 0, ne, kc), l = lower_bound_i(q.sc, f, ne, kc + 1);
            if (f == l) continue;                                   // uniform across the CTA
            const int pq0 = q.pq[f], npq = q.pq[l] - pq0;
            // stage 1: R of every primitive quartet of the sub-chunk
            for (int w = threadIdx.x; w < npq; w += blockDim.x) {
                const int i = lower_bound_i(q.pq, f, l + 1, pq0 + w + 1) - 1;   // last entry with pq <= pq0 + w
                const int rem = pq0 + w - q.pq[i];
                const int ik = rem / nbp, ib = rem - ik * nbp;
                const int P2 = qa.sorted[q.pos[i]];
                stage_r<L>(st, ib, qa.pv.rec + (qa.pv.slot[P2] + ik) * PPW, Rbuf + (size_t)w * NH);
            }
            __syncthreads();
            // stage 2: the column items of the sub-chunk, column-major as in ket_items
            const int nsc = l - f;
            const int items = nsc * nper;
            int it = static_cast<int>(threadIdx.x) - rot;
            if (it < 0) it += blockDim.x;
            for (; it < items; it += blockDim.x) {
                const int i = f + it % nsc;
                work(q.pos[i], it / nsc, Rbuf + (size_t)(q.pq[i] - pq0) * NH);
            }
            rot = (rot + items) % static_cast<int>(blockDim.x);
            __syncthreads();
        }
    }
}

// The ket pairs of class CY for bra position spos whose work falls in the
// chunk's window [w0, w1).
template <int CX, int CY, int NS, bool KGLOBAL, typename RT>
__device__ __forceinline__ void jk_ket_class(const JKArgs& a, const BraStageT<RT>& st, int spos, double* Jt,
                                             facc* Ksm, KetQueueR& kq, int& rot, RT* Rbuf, int64_t w0,
                                             int64_t w1) {
    using Q = QClass<CX, CY>;
    const double q1 = a.q.sortedQ[spos];
    const double* bm = a.bmax;
    const int nb = a.nblock;
    int64_t acc = 0;
    for (int sub = 0; sub < NSUB; ++sub) {
        const int seg = CY * NSUB + sub;
        int64_t kb, ke;
        ket_range<RT>(a.q, seg, spos, kb, ke);
        if (ke <= kb) continue;
        const int64_t wk = ket_work<CX, CY>(sub) * st.nbp;
        int64_t k0, k1;
        window_kets(w0, w1, acc, wk, ke - kb, k0, k1);
        acc += (ke - kb) * wk;
        if (k1 <= k0) continue;
        // difference densities: density-weighted test on the six block pairs
        auto keep = [&](int pos) {
            if (!bm) return true;
            const int P2 = a.q.sorted[pos];
            const int C = a.q.pv.pa_blk[P2], Dd = a.q.pv.pb_blk[P2];
            const double dm = fmax(fmax(bm[st.A * nb + st.B], bm[C * nb + Dd]),
                                   fmax(fmax(bm[st.A * nb + C], bm[st.A * nb + Dd]),
                                        fmax(bm[st.B * nb + C], bm[st.B * nb + Dd])));
            return q1 * a.q.sortedQ[pos] * dm >= a.dthr;
        };
        // contraction groups that the segment's ket pairs actually carry
        const int nkg = seg_groups<Q::KG, Q::NKG>(sub);
        auto digest = [&](int P2, int C, int Dd, int ic, int id, int kg, const RT (&v)[Q::NROW][Q::KG]) {
            if constexpr (sizeof(RT) == sizeof(double)) {
                jk_digest_column<CX, CY, NS, KGLOBAL>(a, st, P2, C, Dd, ic, id, kg, v, Jt, Ksm);
            } else {
                // FP32 quartets: digested (accumulated) in FP64
                double vd[Q::NROW][Q::KG];
#pragma unroll
                for (int r = 0; r < Q::NROW; ++r)
#pragma unroll
                    for (int k = 0; k < Q::KG; ++k) vd[r][k] = static_cast<double>(v[r][k]);
                jk_digest_column<CX, CY, NS, KGLOBAL>(a, st, P2, C, Dd, ic, id, kg, vd, Jt, Ksm);
            }
        };
        // item r = (contraction group, bra-primitive split, column block)
        const int nsp = bra_splits(st.nbp, sub, a.item_pq);
        auto work = [&](int pos, int r, const RT* Rs) {
            const int kg = r % nkg, sp = (r / nkg) % nsp, cd = r / (nkg * nsp);
            const int ib0 = st.nbp * sp / nsp, ib1 = st.nbp * (sp + 1) / nsp;
            const int P2 = a.q.sorted[pos];
            const int C = a.q.pv.pa_blk[P2], Dd = a.q.pv.pb_blk[P2];
            const double* rk = a.q.pv.rec + a.q.pv.slot[P2] * PPW;
            if constexpr (Q::CBLK) {
                // item = the NC columns of one id
                RT v[Q::NC][Q::NROW][Q::KG];
                eri_cols_ket_outer<CX, CY, RT>(st, rk, a.q.pv.npp[P2], cd, kg, v, ib0, ib1);
#pragma unroll
                for (int ic = 0; ic < Q::NC; ++ic) digest(P2, C, Dd, ic, cd, kg, v[ic]);
            } else {
                RT v[Q::NROW][Q::KG];
                eri_column<CX, CY, RT, Q::RSMEM>(st, rk, a.q.pv.npp[P2], cd / Q::ND, cd % Q::ND, kg, v, Rs, ib0,
                                                 ib1);
                digest(P2, C, Dd, cd / Q::ND, cd % Q::ND, kg, v);
            }
        };
        const int j0 = a.q.seg_start[seg] + static_cast<int>(kb + k0);
        if constexpr (Q::RSMEM) {
            ket_items_r<Q::L>(Q::NITEM * nkg * nsp, j0, k1 - k0, kq, rot, st, a.q, Rbuf, keep, work);
        } else {
            ket_items(Q::NITEM * nkg * nsp, j0, k1 - k0, kq, rot, keep,
                      [&](int pos, int r) { work(pos, r, static_cast<const RT*>(nullptr)); });
        }
    }
}

template <int CX, int NS>
struct JKKernel {
    using Q0 = QClass<CX, 0>;
    static constexpr int NROW = Q0::NROW;
    static constexpr int NF = Q0::KA * Q0::NA + Q0::KB * Q0::NB;
    static constexpr int ESIZE = BraE<Q0::LA, Q0::LB, 0>::SIZE;
    // bra classes above ss: one kernel per ket class, so that each kernel
    // holds the code of one ket class only and the CTAs resident on an SM
    // share their instructions; dd bras accumulate K in global memory
    static constexpr bool SPLIT = CX >= 1;
    static constexpr int NY = SPLIT ? CX + 1 : 1;
    static constexpr bool KGLOBAL = CX == 5;
    static constexpr int KROWS = KGLOBAL ? 0 : NS * NF;
};

// Dynamic shared memory: K rows [NS][NF][nao] (unless KGLOBAL), per-thread
// J_ab slots [NS][NROW][blockDim], bra stage.
constexpr int JK_THREADS = 128;

// RT = double: the FP64 quartets; RT = float: the FP32 quartets of the
// mixed-precision path (their J/K contributions still accumulate in FP64).
// YK = ket class of this kernel (-1: the ss bras, whose only ket class is ss).
// Persistent: a CTA runs chunks of the launch's work plan until it is used up.
#ifndef AIMD_JK_MINB
#define AIMD_JK_MINB 1
#endif
template <int CX, int NS, typename RT, int YK>
__global__ void __launch_bounds__(JK_THREADS, AIMD_JK_MINB) jk_bra_kernel(JKArgs a) {
    using KK = JKKernel<CX, NS>;
    using Q0 = QClass<CX, 0>;
    constexpr int Y = YK < 0 ? 0 : YK;      // the unsplit kernel (CX = 0) has one ket class too
    static_assert(YK >= 0 || CX == 0, "bra classes above ss are split by ket class");
    extern __shared__ double smem[];
    const int n = a.q.nao;
    const size_t nn = (size_t)n * n;
    const int krows = a.kglobal ? 0 : KK::KROWS;
    facc* Ksm = reinterpret_cast<facc*>(smem);
    double* Jt = smem + (size_t)krows * n;
    RT* Rbuf = reinterpret_cast<RT*>(Jt + NS * KK::NROW * JK_THREADS);
    RT* Esm = Rbuf + a.rbuf;
    __shared__ BraStageT<RT> st;
    __shared__ KetQueueR kq;
    __shared__ int sh[2];
    const int nbra = a.q.cls_start[CX + 1] - a.q.cls_start[CX];
    const int total = a.plan.off[nbra];
    for (;;) {
        int c, b;
        next_chunk(a.plan, nbra, sh, c, b);
        if (c >= total) break;                                  // uniform: c is shared
        const int spos = a.q.cls_start[CX] + b;
        const int nch = a.plan.off[b + 1] - a.plan.off[b], j = c - a.plan.off[b];
        const int64_t W = bra_work<CX, Y, RT>(a.q, spos);
        if (threadIdx.x == 0) load_stage(a.q, a.q.sorted[spos], st, Esm);
        for (int i = threadIdx.x; i < krows * n + NS * KK::NROW * JK_THREADS; i += blockDim.x) smem[i] = 0.0;
        __syncthreads();
        stage_bra_e<Q0::LA, Q0::LB, 0>(st);
        __syncthreads();
        int rot = 0;
        jk_ket_class<CX, Y, NS, KK::KGLOBAL, RT>(a, st, spos, Jt, Ksm, kq, rot, Rbuf, chunk_edge(W, j, nch),
                                                 chunk_edge(W, j + 1, nch));
        __syncthreads();
        // flush J_ab: one thread per (set, row) sums the per-thread slots
        for (int i = threadIdx.x; i < NS * KK::NROW; i += blockDim.x) {
            double val = 0.0;
            for (int t = 0; t < JK_THREADS; ++t) val += Jt[i * JK_THREADS + t];
            if (val == 0.0) continue;
            const int s = i / KK::NROW, r = i % KK::NROW;
            const int kab = r / Q0::NAB, ab = r % Q0::NAB;
            const int ka = kab / st.nB, kb = kab % st.nB;
            const int m = st.oA + ka * Q0::NA + ab / Q0::NB, nb_ = st.oB + kb * Q0::NB + ab % Q0::NB;
            fadd(a.J + s * nn + (size_t)m * n + nb_, val, __ldg(a.fix));
        }
        // flush K rows
        if (krows > 0) {
            constexpr int NFA = Q0::KA * Q0::NA;
            for (int i = threadIdx.x; i < krows * n; i += blockDim.x) {
                const facc val = Ksm[i];
                if (val == 0) continue;
                const int col = i % n, f = (i / n) % KK::NF, s = i / (n * KK::NF);
                const int row = f < NFA ? st.oA + f : st.oB + (f - NFA);
                atomicAdd(a.K + s * nn + (size_t)row * n + col, val);     // integer: order-independent
            }
        }
        __syncthreads();
    }
}

// Elements of the staged-R buffer of the (CX, YK) kernel (0 unless two-stage).
template <int CX, int YK, typename RT>
size_t jk_rbuf_elems(int max_bra_prims, int max_ket_prims) {
    if constexpr (YK >= 0) {
        using Q = QClass<CX, YK>;
        if constexpr (Q::RSMEM) return rsmem_bytes<Q::L, RT>(max_bra_prims, max_ket_prims) / sizeof(RT);
    }
    return 0;
}

template <int CX, int NS, typename RT>
size_t jk_smem_bytes(int nao, int max_bra_prims, size_t rbuf_elems, bool kglobal) {
    using KK = JKKernel<CX, NS>;
    const size_t krows = kglobal ? 0 : KK::KROWS;
    return sizeof(double) * (krows * nao + (size_t)NS * KK::NROW * JK_THREADS) +
           sizeof(RT) * (rbuf_elems + (size_t)max_bra_prims * (KK::ESIZE + SBW));
}

// ---------------------------------------------------------- Schwarz

// Q[P] = max_ab |(ab|ab)|^(1/2) (the reference's _schwarz_kernel,
// aimd/qc/integrals.py:864-883): one CTA per pair, one thread per column.
template <int CX>
__global__ void __launch_bounds__(64) schwarz_kernel(QuartetArgs a, const int* pairs_of_class, double* Qout) {
    using Q = QClass<CX, CX>;
    extern __shared__ double smem[];
    __shared__ BraStage st;
    __shared__ unsigned long long qmax;
    const int P = pairs_of_class[blockIdx.x];
    if (threadIdx.x == 0) {
        load_stage(a, P, st, smem);
        qmax = 0ull;
    }
    __syncthreads();
    stage_bra_e<Q::LA, Q::LB, 0>(st);
    __syncthreads();
    for (int cd = threadIdx.x; cd < Q::NCD; cd += blockDim.x) {
        static_assert(Q::KG == Q::KCD, "diagonal quartets keep all contraction combinations in one item");
        double v[Q::NROW][Q::KCD];
        eri_column<CX, CX>(st, st.rec, st.nbp, cd / Q::ND, cd % Q::ND, 0, v, static_cast<const double*>(nullptr), 0,
                           st.nbp);
        double m = 0.0;
#pragma unroll
        for (int ka = 0; ka < Q::KA; ++ka)
#pragma unroll
            for (int kb = 0; kb < Q::KB; ++kb) {
                if (ka >= st.nA || kb >= st.nB) continue;
                const int kk = ka * st.nB + kb;
#pragma unroll
                for (int r = 0; r < Q::NROW; ++r)
                    if (r == kk * Q::NAB + cd) m = fmax(m, fabs(v[r][kk]));
            }
        atomicMax(&qmax, (unsigned long long)__double_as_longlong(m));   // m >= 0: bit order = value order
    }
    __syncthreads();
    if (threadIdx.x == 0) Qout[P] = sqrt(__longlong_as_double((long long)qmax));
}

}  // namespace hf
