// Integral-direct two-electron gradient 1/2 sum Gamma d(mn|ls)/dR.
//
// Same decomposition as the J/K build: one CTA per bra block pair, one
// thread item per (ket pair, ket component pair cd). The quartet list is
// enumerated at thr / Gamma_bound, so every quartet the exact test can keep
// is visited; each item applies the reference's test Q1 Q2 max|Gamma| < thr
// (aimd/qc/integrals.py:1329) to its column of Gamma.
//
//   Gamma_{mnls} = deg [Dc_mn Dc_ls - k/2 sum_x (Dx_ml Dx_ns + Dx_ms Dx_nl)],
//   deg = 1/2 x (2 if A != B) x (2 if C != D) x (2 if P1 != P2)
// (aimd/qc/integrals.py:1298-1328). Centres A and B: shifted bra Hermite
// expansions d/dA_x -> 2a E^{i+1,j} - i E^{i-1,j} with R up to L + 1 (the
// reference's _grad_pass, :1049-1244). Centre C: the same identity on the
// ket expansion, contracted with the bra-transformed Gamma. Centre D:
// translational invariance, -(A + B + C), per column.
#pragma once
#include "hf_eri.cuh"

namespace hf {

struct GradArgs {
    QuartetArgs q;
    const double* Dc;       // [nao][nao] symmetric
    const double* Dx;       // [nx][nao][nao] symmetric
    int nx;
    double kfac;
    double thr;             // exact screening threshold on Q1 Q2 max|Gamma|
    facc* grad;             // [natm][3] (fixed point, FIX_G)
    int natm;
    size_t rbuf;            // elements of the kernel's staged-R buffer (set per launch)
    const double* bmc;      // [nblock][nblock] max |Dc| per block pair
    const double* bmx;      // [nblock][nblock] max over x of |Dx| per block pair (nx > 0)
    int nblock;
    WorkPlan plan;          // chunks of the launch (set per launch)
    int item_pq;            // primitive quartets per split column item (launch shape)
};

constexpr int GRAD_THREADS = 128;

// Two-stage items (R_tuv to L + 1 staged per primitive quartet) for the
// gradient of class pair (CX, CY): the same classes as the J/K build.
template <int CX, int CY>
constexpr bool grad_rsmem() { return QClass<CX, CY>::RSMEM; }

// The other classes keep each thread's R_tuv (to L + 1) in a shared-memory
// column while its passes run, where the columns of the CTA take at most
// 96 KB (two CTAs per SM): R to L + 1 is the largest array of the
// gradient body, and in registers it pushes the body into local memory.
template <int CX, int CY, typename RT>
constexpr bool grad_rcol() {
    return !grad_rsmem<CX, CY>() && nherm(QClass<CX, CY>::L + 1) * sizeof(RT) * GRAD_THREADS <= 96 * 1024;
}

// Bra derivative coefficients of one primitive pair, per direction d:
//   k = 0 (centre A): 2a E^{i+1,j}_t - i E^{i-1,j}_t
//   k = 1 (centre B): 2b E^{i,j+1}_t - j E^{i,j-1}_t
// for i <= LA, j <= LB, t <= LA + LB + 1, staged once per CTA so that the
// per-column derivative pass reads one value instead of building it.
template <int LA, int LB>
struct BraD {
    static constexpr int I = LA + 1, J = LB + 1, T = LA + LB + 2;
    static constexpr int SIZE = 2 * 3 * I * J * T;
    __device__ static int at(int k, int d, int i, int j, int t) { return (((k * 3 + d) * I + i) * J + j) * T + t; }
};

template <int LA, int LB, typename RT>
__device__ __forceinline__ void stage_bra_d(const BraStageT<RT>& st) {
    using BE = BraE<LA, LB, 1>;
    using BD = BraD<LA, LB>;
    for (int w = threadIdx.x; w < st.nbp * BD::SIZE; w += blockDim.x) {
        const int ib = w / BD::SIZE, r = w % BD::SIZE;
        const int t = r % BD::T, j = (r / BD::T) % BD::J, i = (r / (BD::T * BD::J)) % BD::I;
        const int d = (r / (BD::T * BD::J * BD::I)) % 3, k = r / (BD::T * BD::J * BD::I * 3);
        const RT* E = st.E + (size_t)ib * BE::SIZE;
        const RT* sb = st.SB + (size_t)ib * SBW;
        RT v;
        if (k == 0) v = RT(2) * sb[5] * E[BE::at(d, i + 1, j, t)] - (i > 0 ? i * E[BE::at(d, i - 1, j, t)] : RT(0));
        else v = RT(2) * sb[6] * E[BE::at(d, i, j + 1, t)] - (j > 0 ? j * E[BE::at(d, i, j - 1, t)] : RT(0));
        st.D[(size_t)ib * BD::SIZE + r] = v;
    }
}

// For runtime (i, j): row[t] = E^{ij}_t and drow[t] = 2c E^{i+1,j}_t - i E^{i-1,j}_t
// (the d/dC_x expansion), selected by predicated copies.
template <int LC, int LD, typename RT>
__device__ __forceinline__ void ket_deriv_rows(const RT (&e)[LC + 2][LD + 1][LC + LD + 2], int i, int j, RT c,
                                               RT (&row)[LC + LD + 2], RT (&drow)[LC + LD + 2]) {
#pragma unroll
    for (int t = 0; t <= LC + LD + 1; ++t) row[t] = drow[t] = RT(0);
#pragma unroll
    for (int ii = 0; ii <= LC; ++ii)
#pragma unroll
        for (int jj = 0; jj <= LD; ++jj)
            if (ii == i && jj == j)
#pragma unroll
                for (int t = 0; t <= LC + LD + 1; ++t) {
                    row[t] = t <= LC + LD ? e[ii][jj][t] : RT(0);
                    drow[t] = RT(2) * c * e[ii + 1][jj][t] - (ii > 0 ? ii * e[ii > 0 ? ii - 1 : 0][jj][t] : RT(0));
                }
}

// Primitive loops of one gradient column with the bra-side work hoisted out
// of the ket primitives: bra primitives outer; per bra primitive the
// C-pass weights Y[kk]_h = sum_ab f_ab C_ab Gamma[ab][kk] E^{ab}_h (bra
// only) are formed once, the ket primitives inner accumulate the ket step
// Xs[kk]_h = sum_ik c_ik[kk] pref sum_box(cd) (-1)^|k| E^{cd}_k R_{h+k}
// (h to LAB + 1) and the C pass, and the bra pass for centres A and B runs
// once per bra primitive on Xs (it is linear in the ket step). Same sums as
// the per-primitive-quartet order, regrouped.
template <int CX, int CY, typename RT, bool RS>
__device__ __forceinline__ void grad_prims_hoisted(const BraStageT<RT>& st, const RT (&Gr)[QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                                   const double* __restrict__ rk, int nkp, int ic, int id, int kg,
                                                   RT (&dA)[3], RT (&dB)[3], RT (&dC)[3], const RT* __restrict__ Rs,
                                                   RT* Rcol, int ib0, int ib1) {
    using Q = QClass<CX, CY>;
    using BE = BraE<Q::LA, Q::LB, 1>;
    using BD = BraD<Q::LA, Q::LB>;
    constexpr int LA = Q::LA, LB = Q::LB, LC = Q::LC, LD = Q::LD, LAB = Q::LAB, LCD = Q::LCD, L = Q::L + 1;
    constexpr int NH1 = nherm(LAB + 1);
    constexpr int KG = Q::KG;
    constexpr int UH = L >= 4 ? 1 : 16;     // rolled Hermite loops: smaller code (instruction fetch)
    constexpr int UW = L >= 5 ? 1 : 16;
    const int cx = cart_x(LC, ic), cy = cart_y(LC, ic), cz = cart_z(LC, ic);
    const int dx = cart_x(LD, id), dy = cart_y(LD, id), dz = cart_z(LD, id);
    const RT fcd = cart_norm(cx, cy, cz) * cart_norm(dx, dy, dz);
    for (int ib = ib0; ib < ib1; ++ib) {
        const RT* sb = st.SB + ib * SBW;
        const RT* E = st.E + (size_t)ib * BE::SIZE;
        const RT* Db = st.D + (size_t)ib * BD::SIZE;
        // Gamma of row ab contracted with this bra primitive's coefficients and f_ab
        auto gq = [&](int ia, int jb, int kk) {
            const RT fab = cart_norm(cart_x(LA, ia), cart_y(LA, ia), cart_z(LA, ia)) *
                           cart_norm(cart_x(LB, jb), cart_y(LB, jb), cart_z(LB, jb));
            RT s = RT(0);
#pragma unroll
            for (int kab = 0; kab < Q::KAB; ++kab) s += sb[8 + kab] * Gr[kab * Q::NAB + ia * Q::NB + jb][kk];
            return s * fab;
        };
        RT Y[KG][Q::NHB];
#pragma unroll
        for (int kk = 0; kk < KG; ++kk)
#pragma unroll
            for (int h = 0; h < Q::NHB; ++h) Y[kk][h] = RT(0);
#pragma unroll UH
        for (int ia = 0; ia < Q::NA; ++ia) {
            const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
#pragma unroll
            for (int jb = 0; jb < Q::NB; ++jb) {
                const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                RT g[KG];
#pragma unroll
                for (int kk = 0; kk < KG; ++kk) g[kk] = gq(ia, jb, kk);
#pragma unroll
                for (int t = 0; t <= ax + bx; ++t)
#pragma unroll
                    for (int u = 0; u <= ay + by; ++u) {
                        const RT e01 = E[BE::at(0, ax, bx, t)] * E[BE::at(1, ay, by, u)];
#pragma unroll
                        for (int w = 0; w <= az + bz; ++w) {
                            const RT e = e01 * E[BE::at(2, az, bz, w)];
#pragma unroll
                            for (int kk = 0; kk < KG; ++kk) Y[kk][hidx(t, u, w)] += g[kk] * e;
                        }
                    }
            }
        }
        RT Xs[KG][NH1];
#pragma unroll
        for (int kk = 0; kk < KG; ++kk)
#pragma unroll
            for (int h = 0; h < NH1; ++h) Xs[kk][h] = RT(0);
        for (int ik = 0; ik < nkp; ++ik) {
            const KetRecT<RT> k = load_ket<RT>(rk + (size_t)ik * PPW);
            const RT ec = k.a, q = ec + k.b, oo2q = RT(0.5) / q;
            RT ex[LCD + 2], ey[LCD + 2], ez[LCD + 2], gx[LCD + 2], gy[LCD + 2], gz[LCD + 2];
            {
                RT e[LC + 2][LD + 1][LCD + 2];
                hermite_e<LC + 1, LD>(k.QAx, k.QBx, oo2q, k.K, e);
                ket_deriv_rows<LC, LD>(e, cx, dx, ec, ex, gx);
                hermite_e<LC + 1, LD>(k.QAy, k.QBy, oo2q, RT(1), e);
                ket_deriv_rows<LC, LD>(e, cy, dy, ec, ey, gy);
                hermite_e<LC + 1, LD>(k.QAz, k.QBz, oo2q, RT(1), e);
                ket_deriv_rows<LC, LD>(e, cz, dz, ec, ez, gz);
            }
            RT ck[KG];
#pragma unroll
            for (int i = 0; i < KG; ++i) {
                RT c = k.c[0];
#pragma unroll
                for (int j = 1; j < Q::KCD; ++j)
                    if (j == kg * KG + i) c = k.c[j];
                ck[i] = c * fcd;
            }
            auto body = [&](const auto& R, RT scale) {
                RT sc[KG];
#pragma unroll
                for (int kk = 0; kk < KG; ++kk) sc[kk] = scale * ck[kk];
                // ket step for the bra pass, accumulated over the ket primitives
#pragma unroll UH
                for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll UH
                    for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll UW
                        for (int w = 0; w <= LAB + 1 - t - u; ++w) {
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
                                        s += ((v2 & 1) ? -exy * ez[v2] : exy * ez[v2]) * R[hidx(t + t2, u + u2, w + v2)];
                                    }
                                }
                            }
#pragma unroll
                            for (int kk = 0; kk < KG; ++kk) Xs[kk][hidx(t, u, w)] += sc[kk] * s;
                        }
                // C pass: dC_d += sum_k dE^{cd}_{d,k} Z_k with Z_k = (-1)^|k| sum_h Y_h R_{h+k},
                // k over the ket box widened by one in at most one direction
                // (the rows are zero beyond their box): Z is shared by the
                // three directions
#pragma unroll
                for (int t2 = 0; t2 <= LCD + 1; ++t2) {
                    if (t2 > cx + dx + 1) continue;
#pragma unroll
                    for (int u2 = 0; u2 <= LCD + 1; ++u2) {
                        if (u2 > cy + dy + 1) continue;
#pragma unroll
                        for (int v2 = 0; v2 <= LCD + 1; ++v2) {
                            if (v2 > cz + dz + 1) continue;
                            if ((t2 > cx + dx) + (u2 > cy + dy) + (v2 > cz + dz) > 1) continue;
                            RT z[KG];
#pragma unroll
                            for (int kk = 0; kk < KG; ++kk) z[kk] = RT(0);
#pragma unroll UH
                            for (int t = 0; t <= LAB; ++t)
#pragma unroll UH
                                for (int u = 0; u <= LAB - t; ++u)
#pragma unroll UW
                                    for (int w = 0; w <= LAB - t - u; ++w) {
                                        const RT r = R[hidx(t + t2, u + u2, w + v2)];
#pragma unroll
                                        for (int kk = 0; kk < KG; ++kk) z[kk] += Y[kk][hidx(t, u, w)] * r;
                                    }
                            RT zs = RT(0);
#pragma unroll
                            for (int kk = 0; kk < KG; ++kk) zs += sc[kk] * z[kk];
                            if ((t2 + u2 + v2) & 1) zs = -zs;
                            dC[0] += gx[t2] * ey[u2] * ez[v2] * zs;
                            dC[1] += ex[t2] * gy[u2] * ez[v2] * zs;
                            dC[2] += ex[t2] * ey[u2] * gz[v2] * zs;
                        }
                    }
                }
            };
            if constexpr (RS) {
                body(Rs + (size_t)(ik * st.nbp + ib) * nherm(L), RT(1));
            } else {
                const RT p = sb[0];
                const RT rs = rsqrt_t(p + q);
                const RT alpha = p * q * rs * rs;
                const RT pref = RT(TWO_PI_2_5) * sb[1] * (RT(2) * oo2q) * rs;
                RT R[nherm(L)];
                if constexpr (grad_rcol<CX, CY, RT>()) {
                    hermite_r_scaled<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, pref, R);
#pragma unroll
                    for (int i = 0; i < nherm(L); ++i) Rcol[i * GRAD_THREADS] = R[i];
                    body(RColumn<RT, GRAD_THREADS>{Rcol}, RT(1));
                } else {
                    hermite_r<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, R);
                    body(R, pref);
                }
            }
        }
        // bra pass (A, B) on the summed ket step, once per bra primitive
#pragma unroll UH
        for (int ia = 0; ia < Q::NA; ++ia) {
            const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
#pragma unroll
            for (int jb = 0; jb < Q::NB; ++jb) {
                const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                RT g[KG];
#pragma unroll
                for (int kk = 0; kk < KG; ++kk) g[kk] = gq(ia, jb, kk);
#pragma unroll
                for (int t = 0; t <= ax + bx + 1; ++t)
#pragma unroll
                    for (int u = 0; u <= ay + by + 1; ++u)
#pragma unroll
                        for (int w = 0; w <= az + bz + 1; ++w) {
                            const int over = (t > ax + bx) + (u > ay + by) + (w > az + bz);
                            if (over > 1) continue;
                            RT yv = RT(0);
#pragma unroll
                            for (int kk = 0; kk < KG; ++kk) yv += g[kk] * Xs[kk][hidx(t, u, w)];
                            const RT e0 = E[BE::at(0, ax, bx, t)], e1 = E[BE::at(1, ay, by, u)],
                                     e2 = E[BE::at(2, az, bz, w)];
                            const RT y12 = yv * e1 * e2, y02 = yv * e0 * e2, y01 = yv * e0 * e1;
                            dA[0] += y12 * Db[BD::at(0, 0, ax, bx, t)];
                            dA[1] += y02 * Db[BD::at(0, 1, ay, by, u)];
                            dA[2] += y01 * Db[BD::at(0, 2, az, bz, w)];
                            dB[0] += y12 * Db[BD::at(1, 0, ax, bx, t)];
                            dB[1] += y02 * Db[BD::at(1, 1, ay, by, u)];
                            dB[2] += y01 * Db[BD::at(1, 2, az, bz, w)];
                        }
            }
        }
    }
}

// The hoisted order for the d-shell bra classes, where its register
// footprint (Gamma column, Y and the summed ket step per contraction group)
// fits (up to the 127 doubles of the dd bras, whose pairs have one bra
// primitive, so the bra pass runs once per column instead of once per ket
// primitive); the per-primitive-quartet order for the others (measured:
// hoisting the s/p bras, whose pairs have many primitives, was no faster).
template <int CX, int CY, typename RT>
constexpr bool grad_hoist() {
    using Q = QClass<CX, CY>;
    // d-shell bras only (few bra primitives; see eri_column)
    return CX >= 3 && sizeof(RT) * (Q::NROW * Q::KG + Q::KG * (Q::NHB + nherm(Q::LAB + 1))) <= 1100;
}

// One primitive quartet (bra primitive sb/E/Db, ket primitive through its
// column rows ex.. and derivative rows gx..) of one gradient column:
// adds the A, B and C derivative parts. Everything is linear in pref * R.
template <int CX, int CY, typename RT, typename RArr>
__device__ __forceinline__ void grad_pq(const RT* sb, const RT* E, const RT* Db,
                                        const RT (&Gr)[QClass<CX, CY>::NROW][QClass<CX, CY>::KG],
                                        const RT (&ck)[QClass<CX, CY>::KG], int cx, int cy, int cz, int dx, int dy,
                                        int dz, const RT (&ex)[QClass<CX, CY>::LCD + 2],
                                        const RT (&ey)[QClass<CX, CY>::LCD + 2],
                                        const RT (&ez)[QClass<CX, CY>::LCD + 2],
                                        const RT (&gx)[QClass<CX, CY>::LCD + 2],
                                        const RT (&gy)[QClass<CX, CY>::LCD + 2],
                                        const RT (&gz)[QClass<CX, CY>::LCD + 2], const RArr& R, RT pref,
                                        RT (&dA)[3], RT (&dB)[3], RT (&dC)[3]) {
    using Q = QClass<CX, CY>;
    using BE = BraE<Q::LA, Q::LB, 1>;
    using BD = BraD<Q::LA, Q::LB>;
    constexpr int LA = Q::LA, LB = Q::LB, LAB = Q::LAB, LCD = Q::LCD, L = Q::L + 1;
    constexpr int NH1 = nherm(LAB + 1);
    constexpr int UH = L >= 5 ? 1 : 16;      // rolled outer Hermite loops for large classes
    constexpr int UW = L >= 7 ? 1 : 16;      // and the inner one for the largest (compile time)

            // Gamma contracted with this bra primitive's coefficients and f_ab,
            // then summed over the ket contractions: gq[ab] = sum_kk gb[ab][kk] ck[kk]
            RT gq[Q::NAB];
#pragma unroll
            for (int ia = 0; ia < Q::NA; ++ia)
#pragma unroll
                for (int jb = 0; jb < Q::NB; ++jb) {
                    const RT fab = cart_norm(cart_x(LA, ia), cart_y(LA, ia), cart_z(LA, ia)) *
                                       cart_norm(cart_x(LB, jb), cart_y(LB, jb), cart_z(LB, jb));
                    const int ab = ia * Q::NB + jb;
                    RT s = 0.0;
#pragma unroll
                    for (int kab = 0; kab < Q::KAB; ++kab)
#pragma unroll
                        for (int kk = 0; kk < Q::KG; ++kk) s += sb[8 + kab] * Gr[kab * Q::NAB + ab][kk] * ck[kk];
                    gq[ab] = s * fab * pref;
                }
            // bra pass (A, B): sum_ab gq[ab] sum_{h in dbox(ab)} dE_h Xb_h,
            // Xb_h = sum_{k in box(cd)} (-1)^|k| E^{cd}_k R_{h+k}
            RT Xb[NH1];
#pragma unroll UH
            for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll UH
                for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll UW
                    for (int w = 0; w <= LAB + 1 - t - u; ++w) {
                        RT s = 0.0;
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
                                    s += ((v2 & 1) ? -exy * ez[v2] : exy * ez[v2]) * R[hidx(t + t2, u + u2, w + v2)];
                                }
                            }
                        }
                        Xb[hidx(t, u, w)] = s;
                    }
            // C pass: Y_h = sum_ab gq[ab] E^{ab}_h (h <= LAB), then
            // dC_d += sum_h Y_h sum_k (-1)^|k| dE^{cd}_{d,k} R_{h+k} (in this
            // order the per-direction form spills less than the Z form of
            // the hoisted order)
            RT Y[Q::NHB];
#pragma unroll
            for (int h = 0; h < Q::NHB; ++h) Y[h] = 0.0;
#pragma unroll UH
            for (int ia = 0; ia < Q::NA; ++ia) {
                const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
#pragma unroll
                for (int jb = 0; jb < Q::NB; ++jb) {
                    const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                    const RT g = gq[ia * Q::NB + jb];
#pragma unroll
                    for (int t = 0; t <= ax + bx + 1; ++t)
#pragma unroll
                        for (int u = 0; u <= ay + by + 1; ++u)
#pragma unroll
                            for (int w = 0; w <= az + bz + 1; ++w) {
                                const int over = (t > ax + bx) + (u > ay + by) + (w > az + bz);
                                if (over > 1) continue;
                                const RT yv = g * Xb[hidx(t, u, w)];
                                const RT e0 = E[BE::at(0, ax, bx, t)], e1 = E[BE::at(1, ay, by, u)],
                                             e2 = E[BE::at(2, az, bz, w)];
                                const RT e12 = e1 * e2, e02 = e0 * e2, e01 = e0 * e1;
                                if (over == 0) Y[hidx(t, u, w)] += g * e01 * e2;
                                const RT y12 = yv * e12, y02 = yv * e02, y01 = yv * e01;
                                dA[0] += y12 * Db[BD::at(0, 0, ax, bx, t)];
                                dA[1] += y02 * Db[BD::at(0, 1, ay, by, u)];
                                dA[2] += y01 * Db[BD::at(0, 2, az, bz, w)];
                                dB[0] += y12 * Db[BD::at(1, 0, ax, bx, t)];
                                dB[1] += y02 * Db[BD::at(1, 1, ay, by, u)];
                                dB[2] += y01 * Db[BD::at(1, 2, az, bz, w)];
                            }
                }
            }
#pragma unroll UH
            for (int t = 0; t <= LAB; ++t)
#pragma unroll UH
                for (int u = 0; u <= LAB - t; ++u)
#pragma unroll UW
                    for (int w = 0; w <= LAB - t - u; ++w) {
                        const RT yv = Y[hidx(t, u, w)];
                        // one direction d at a time (one accumulator live)
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            RT sd = 0.0;
#pragma unroll
                            for (int t2 = 0; t2 <= LCD + 1; ++t2) {
                                if (t2 > cx + dx + (d == 0)) continue;
#pragma unroll
                                for (int u2 = 0; u2 <= LCD + 1; ++u2) {
                                    if (u2 > cy + dy + (d == 1)) continue;
                                    const RT fxy = (d == 0 ? gx[t2] : ex[t2]) * (d == 1 ? gy[u2] : ey[u2]);
#pragma unroll
                                    for (int v2 = 0; v2 <= LCD + 1; ++v2) {
                                        if (v2 > cz + dz + (d == 2)) continue;
                                        const RT r = ((t2 + u2 + v2) & 1) ? -R[hidx(t + t2, u + u2, w + v2)]
                                                                              : R[hidx(t + t2, u + u2, w + v2)];
                                        sd += fxy * (d == 2 ? gz[v2] : ez[v2]) * r;
                                    }
                                }
                            }
                            dC[d] += yv * sd;
                        }
                    }
}

// Gradient contribution of one column; adds A, B parts to gab and C, D
// parts to the shared accumulator gsh[natm][3]. RS: pref * R_tuv (to L + 1)
// of the ket pair's primitive quartets staged in Rs ([ik][ib][NH(L + 1)]).
template <int CX, int CY, typename RT, bool RS = false>
__device__ __forceinline__ void grad_column(const GradArgs& a, const BraStageT<RT>& st, int P2, double QQ, int ic,
                                            int id, int kg, double (&gab)[6], facc* gsh,
                                            const RT* __restrict__ Rs, RT* Rcol, int ib0, int ib1) {
    using Q = QClass<CX, CY>;
    using BE = BraE<Q::LA, Q::LB, 1>;
    using BD = BraD<Q::LA, Q::LB>;
    constexpr int LA = Q::LA, LB = Q::LB, LC = Q::LC, LD = Q::LD, LAB = Q::LAB, LCD = Q::LCD, L = Q::L + 1;
    constexpr int NH1 = nherm(LAB + 1);
    constexpr int UH = L >= 5 ? 1 : 16;      // rolled outer Hermite loops for large classes
    constexpr int UW = L >= 7 ? 1 : 16;      // and the inner one for the largest (compile time)
    const BlockView& bv = a.q.bv;
    const int C = a.q.pv.pa_blk[P2], Dd = a.q.pv.pb_blk[P2];
    const int aC = bv.atom[C], aD = bv.atom[Dd];
    if (st.aA == st.aB && st.aB == aC && aC == aD) return;          // one-centre: invariant
    const int nC = bv.ncon[C], nD = bv.ncon[Dd], oC = bv.ao[C], oD = bv.ao[Dd];
    const int n = a.q.nao;
    const size_t nn = (size_t)n * n;
    const double deg = 0.5 * (st.A != st.B ? 2.0 : 1.0) * (C != Dd ? 2.0 : 1.0) * (st.P1 != P2 ? 2.0 : 1.0);
    // Gamma column
    double G[Q::NROW][Q::KG];
    double gmax = 0.0;
#pragma unroll
    for (int kk = 0; kk < Q::KG; ++kk) {
        const int kq = kg * Q::KG + kk;
        const bool cv = kq < nC * nD;
        const int kc = cv ? kq / nD : 0, kd = cv ? kq % nD : 0;
        const size_t l = oC + kc * Q::NC + ic, sg = oD + kd * Q::ND + id;
#pragma unroll
        for (int r = 0; r < Q::NROW; ++r) {
            const int kab = r / Q::NAB, ab = r % Q::NAB, ka = kab / st.nB, kb = kab % st.nB;
            double val = 0.0;
            if (cv && kab < st.nA * st.nB) {
                const size_t m = st.oA + ka * Q::NA + ab / Q::NB, nb_ = st.oB + kb * Q::NB + ab % Q::NB;
                val = __ldg(a.Dc + m * n + nb_) * __ldg(a.Dc + l * n + sg);
                for (int x = 0; x < a.nx; ++x) {
                    const double* X = a.Dx + x * nn;
                    val -= 0.5 * a.kfac * (__ldg(X + m * n + l) * __ldg(X + nb_ * n + sg) +
                                           __ldg(X + m * n + sg) * __ldg(X + nb_ * n + l));
                }
                val *= deg;
            }
            G[r][kk] = val;
            gmax = fmax(gmax, fabs(val));
        }
    }
    if (QQ == 0.0 || QQ * gmax < a.thr) return;
    // the Gamma column in the arithmetic type of the quartet
    RT Gr[Q::NROW][Q::KG];
#pragma unroll
    for (int r = 0; r < Q::NROW; ++r)
#pragma unroll
        for (int kk = 0; kk < Q::KG; ++kk) Gr[r][kk] = static_cast<RT>(G[r][kk]);
    RT dA[3] = {0.0, 0.0, 0.0}, dB[3] = {0.0, 0.0, 0.0}, dC[3] = {0.0, 0.0, 0.0};
    if constexpr (grad_hoist<CX, CY, RT>()) {
        grad_prims_hoisted<CX, CY, RT, RS>(st, Gr, a.q.pv.rec + a.q.pv.slot[P2] * PPW, a.q.pv.npp[P2], ic, id, kg,
                                           dA, dB, dC, Rs, Rcol, ib0, ib1);
    } else {
    const int cx = cart_x(LC, ic), cy = cart_y(LC, ic), cz = cart_z(LC, ic);
    const int dx = cart_x(LD, id), dy = cart_y(LD, id), dz = cart_z(LD, id);
    const RT fcd = cart_norm(cx, cy, cz) * cart_norm(dx, dy, dz);
    const double* rk = a.q.pv.rec + a.q.pv.slot[P2] * PPW;
    const int nkp = a.q.pv.npp[P2];
    for (int ik = 0; ik < nkp; ++ik) {
        const KetRecT<RT> k = load_ket<RT>(rk + (size_t)ik * PPW);
        const RT ec = k.a, q = ec + k.b, oo2q = RT(0.5) / q, iq = RT(2) * oo2q;
        // ket E for this column, and d/dC_d of it (one extra in direction d)
        RT ex[LCD + 2], ey[LCD + 2], ez[LCD + 2], gx[LCD + 2], gy[LCD + 2], gz[LCD + 2];
        {
            RT e[LC + 2][LD + 1][LCD + 2];
            hermite_e<LC + 1, LD>(k.QAx, k.QBx, oo2q, k.K, e);
            ket_deriv_rows<LC, LD>(e, cx, dx, ec, ex, gx);
            hermite_e<LC + 1, LD>(k.QAy, k.QBy, oo2q, RT(1), e);
            ket_deriv_rows<LC, LD>(e, cy, dy, ec, ey, gy);
            hermite_e<LC + 1, LD>(k.QAz, k.QBz, oo2q, RT(1), e);
            ket_deriv_rows<LC, LD>(e, cz, dz, ec, ez, gz);
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
            const RT* E = st.E + (size_t)ib * BE::SIZE;
            const RT* Db = st.D + (size_t)ib * BD::SIZE;
            // everything below is linear in pref * R_tuv (R up to L + 1)
            auto body = [&](const auto& R, RT pref) {
                grad_pq<CX, CY, RT>(sb, E, Db, Gr, ck, cx, cy, cz, dx, dy, dz, ex, ey, ez, gx, gy, gz, R, pref, dA, dB,
                                    dC);
            };
            if constexpr (RS) {
                body(Rs + (size_t)(ik * st.nbp + ib) * nherm(L), RT(1));
            } else {
                const RT p = sb[0];
                const RT rs = rsqrt_t(p + q);
                const RT alpha = p * q * rs * rs;
                const RT pref = RT(TWO_PI_2_5) * sb[1] * iq * rs;
                RT R[nherm(L)];
                if constexpr (grad_rcol<CX, CY, RT>()) {
                    hermite_r_scaled<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, pref, R);
#pragma unroll
                    for (int i = 0; i < nherm(L); ++i) Rcol[i * GRAD_THREADS] = R[i];
                    body(RColumn<RT, GRAD_THREADS>{Rcol}, RT(1));
                } else {
                    hermite_r<L>(alpha, sb[2] - k.Qx, sb[3] - k.Qy, sb[4] - k.Qz, R);
                    body(R, pref);
                }
            }
        }
    }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double da = dA[d], db = dB[d], dc = dC[d];
        gab[d] += da;
        gab[3 + d] += db;
        fadd(gsh + 3 * aC + d, dc, FIX_G);
        fadd(gsh + 3 * aD + d, -(da + db + dc), FIX_G);
    }
}

// Ket pairs pass the queue when the block bound of Gamma over the whole
// block quartet, deg [|Dc|_AB |Dc|_CD + |k|/2 nx (|Dx|_AC |Dx|_BD +
// |Dx|_AD |Dx|_BC)] >= max|Gamma|, can reach the threshold and the quartet
// is not one-centre; the exact per-column test follows in grad_column.

template <int CX, int CY, typename RT>
__device__ __forceinline__ void grad_ket_class(const GradArgs& a, const BraStageT<RT>& st, int spos, double (&gab)[6],
                                               facc* gsh, KetQueueR& kq, int& rot, RT* Rbuf, int64_t w0,
                                               int64_t w1) {
    using Q = QClass<CX, CY>;
    constexpr bool RS = grad_rsmem<CX, CY>();
    const double q1 = a.q.sortedQ[spos];
    const int nb = a.nblock;
    const double xf = 0.5 * fabs(a.kfac) * a.nx;
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
        auto keep = [&](int pos) {
            const int P2 = a.q.sorted[pos];
            const int C = a.q.pv.pa_blk[P2], Dd = a.q.pv.pb_blk[P2];
            const int aC = a.q.bv.atom[C], aD = a.q.bv.atom[Dd];
            if (st.aA == st.aB && st.aB == aC && aC == aD) return false;
            double gb = a.bmc[st.A * nb + st.B] * a.bmc[C * nb + Dd];
            if (a.nx > 0)
                gb += xf * (a.bmx[st.A * nb + C] * a.bmx[st.B * nb + Dd] + a.bmx[st.A * nb + Dd] * a.bmx[st.B * nb + C]);
            const double deg = 0.5 * (st.A != st.B ? 2.0 : 1.0) * (C != Dd ? 2.0 : 1.0) * (st.P1 != P2 ? 2.0 : 1.0);
            return q1 * a.q.sortedQ[pos] * deg * gb >= a.thr;
        };
        const int nkg = seg_groups<Q::KG, Q::NKG>(sub);
        // item r = (contraction group, bra-primitive split, column)
        const int nsp = bra_splits(st.nbp, sub, a.item_pq);
        auto work = [&](int pos, int r, const RT* Rs) {
            const int kg = r % nkg, sp = (r / nkg) % nsp, cd = r / (nkg * nsp);
            grad_column<CX, CY, RT, RS>(a, st, a.q.sorted[pos], q1 * a.q.sortedQ[pos], cd / Q::ND, cd % Q::ND, kg,
                                        gab, gsh, Rs, Rbuf + threadIdx.x, st.nbp * sp / nsp,
                                        st.nbp * (sp + 1) / nsp);
        };
        const int j0 = a.q.seg_start[seg] + static_cast<int>(kb + k0);
        if constexpr (RS) {
            ket_items_r<Q::L + 1>(Q::NCD * nkg * nsp, j0, k1 - k0, kq, rot, st, a.q, Rbuf, keep, work);
        } else {
            ket_items(Q::NCD * nkg * nsp, j0, k1 - k0, kq, rot, keep,
                      [&](int pos, int r) { work(pos, r, static_cast<const RT*>(nullptr)); });
        }
    }
}

// One kernel per (bra class, ket class), persistent: a CTA runs chunks
// (bra pair of class CX, window of its ket pairs of class CY) of the
// launch's work plan until it is used up. Dynamic shared memory: gradient
// accumulator [natm][3] (one per CTA, flushed at the end), staged R, bra E
// tables (+1).
// RT = double: the FP64 quartets; RT = float: the FP32 quartets of the
// mixed-precision path (accumulated in FP64).
#ifndef AIMD_GRAD_MINB
#define AIMD_GRAD_MINB 1
#endif
template <int CX, int CY, typename RT>
__global__ void __launch_bounds__(GRAD_THREADS, AIMD_GRAD_MINB) grad2e_bra_kernel(GradArgs a) {
    using Q0 = QClass<CX, 0>;
    extern __shared__ double smem[];
    facc* gsh = reinterpret_cast<facc*>(smem);
    RT* Rbuf = reinterpret_cast<RT*>(smem + 3 * a.natm);
    RT* Esm = Rbuf + a.rbuf;
    __shared__ BraStageT<RT> st;
    __shared__ KetQueueR kq;
    __shared__ int sh[2];
    const int nbra = a.q.cls_start[CX + 1] - a.q.cls_start[CX];
    const int total = a.plan.off[nbra];
    for (int i = threadIdx.x; i < 3 * a.natm; i += blockDim.x) gsh[i] = 0;
    for (;;) {
        int c, b;
        next_chunk(a.plan, nbra, sh, c, b);                     // (its barrier also orders the zeroing)
        if (c >= total) break;                                  // uniform: c is shared
        const int spos = a.q.cls_start[CX] + b;
        const int nch = a.plan.off[b + 1] - a.plan.off[b], j = c - a.plan.off[b];
        const int64_t W = bra_work<CX, CY, RT>(a.q, spos);
        if (threadIdx.x == 0) {
            load_stage(a.q, a.q.sorted[spos], st, Esm);
            st.D = st.E + (size_t)st.nbp * BraE<Q0::LA, Q0::LB, 1>::SIZE;
        }
        __syncthreads();
        stage_bra_e<Q0::LA, Q0::LB, 1>(st);
        __syncthreads();
        stage_bra_d<Q0::LA, Q0::LB>(st);
        __syncthreads();
        double gab[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int rot = 0;
        grad_ket_class<CX, CY, RT>(a, st, spos, gab, gsh, kq, rot, Rbuf, chunk_edge(W, j, nch),
                                   chunk_edge(W, j + 1, nch));
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (gab[d] != 0.0) fadd(gsh + 3 * st.aA + d, gab[d], FIX_G);
            if (gab[3 + d] != 0.0) fadd(gsh + 3 * st.aB + d, gab[3 + d], FIX_G);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < 3 * a.natm; i += blockDim.x)
        if (gsh[i] != 0) atomicAdd(a.grad + i, gsh[i]);
}

// Elements of the staged-R buffer of the (CX, CY) gradient kernel (the
// two-stage classes), or of its threads' R columns.
template <int CX, int CY, typename RT>
size_t grad_rbuf_elems(int max_bra_prims, int max_ket_prims) {
    if constexpr (grad_rsmem<CX, CY>())
        return rsmem_bytes<QClass<CX, CY>::L + 1, RT>(max_bra_prims, max_ket_prims) / sizeof(RT);
    if constexpr (grad_rcol<CX, CY, RT>()) return (size_t)nherm(QClass<CX, CY>::L + 1) * GRAD_THREADS;
    return 0;
}

template <int CX, typename RT>
size_t grad_smem_bytes(int natm, int max_bra_prims, size_t rbuf_elems) {
    using Q0 = QClass<CX, 0>;
    return sizeof(double) * 3 * (size_t)natm +
           sizeof(RT) * (rbuf_elems + (size_t)max_bra_prims * (BraE<Q0::LA, Q0::LB, 1>::SIZE +
                                                              BraD<Q0::LA, Q0::LB>::SIZE + SBW));
}

}  // namespace hf
