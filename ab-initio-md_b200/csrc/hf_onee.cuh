// One-electron integrals and their nuclear-derivative contractions.
//
// One thread per segmented shell pair (si >= sj), class-templated on
// (l_i, l_j). Overlap-type integrals use t = 0 Hermite coefficients
// (E^{ij}_0 sqrt(pi/p) per direction), kinetic energy the 1-D second
// derivative identity, the dipole E^{ij}_1 + X_PO E^{ij}_0, and the nuclear
// attraction the Hermite Coulomb integrals R_tuv(p, P - C). Derivatives come
// from the Gaussian-centre identity d/dA_x x_A^i = 2a x_A^{i+1} - i x_A^{i-1}
// and dR/dC = -R_{t+1}; translational invariance supplies the second centre.
// (The reference's _overlap_type_kernel, _nuclear_kernel,
// _overlap_kinetic_grad_kernel and _nuclear_grad_kernel,
// aimd/qc/integrals.py:155-501.)
#pragma once
#include "hf_device.cuh"

namespace hf {

struct ShellView {
    int nshell, natm, nao;
    const int* atom;
    const int* l;
    const int* ao;
    const int* p0;      // first primitive
    const int* np;      // primitive count
    const double* exps;
    const double* coefs;
    const double* pos;  // [natm][3]
    const double* charges;
    const int* pair_i;  // shell pairs (si >= sj), grouped by class (li, lj) with li >= lj
    const int* pair_j;
};

// -1/2 <i| d^2/dx^2 |j> from overlap factors e[i][j][0] (j up to J+2 present)
template <int IM, int JM>
__device__ __forceinline__ double kin1d(const double (&e)[IM + 1][JM + 1][IM + JM + 1], int i, int j, double b) {
    double v = -2.0 * b * (2 * j + 1) * e[i][j][0] + 4.0 * b * b * e[i][j + 2][0];
    if (j >= 2) v += j * (j - 1) * e[i][j - 2][0];
    return -0.5 * v;
}

// S, T, dipole (about origin o) and V for shell pairs of class (LI, LJ);
// pairs [p_begin, p_end) of the class-sorted shell-pair list.
template <int LI, int LJ>
__global__ void __launch_bounds__(128) onee_kernel(ShellView sv, int p_begin, int p_end, double ox, double oy,
                                                   double oz, double* S, double* T,
                                                   double* M, double* V) {
    const int ip = p_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (ip >= p_end) return;
    const int si = sv.pair_i[ip], sj = sv.pair_j[ip];
    constexpr int NI = ncart(LI), NJ = ncart(LJ), L = LI + LJ;
    const int ai = sv.atom[si], aj = sv.atom[sj];
    const double Ax = sv.pos[3 * ai], Ay = sv.pos[3 * ai + 1], Az = sv.pos[3 * ai + 2];
    const double Bx = sv.pos[3 * aj], By = sv.pos[3 * aj + 1], Bz = sv.pos[3 * aj + 2];
    const double ABx = Ax - Bx, ABy = Ay - By, ABz = Az - Bz;
    double s[NI][NJ] = {}, t[NI][NJ] = {}, mx[NI][NJ] = {}, my[NI][NJ] = {}, mz[NI][NJ] = {}, vv[NI][NJ] = {};
    const double sqpi = sqrt(PI);
    for (int ka = sv.p0[si]; ka < sv.p0[si] + sv.np[si]; ++ka) {
        const double a = sv.exps[ka];
        for (int kb = sv.p0[sj]; kb < sv.p0[sj] + sv.np[sj]; ++kb) {
            const double b = sv.exps[kb], p = a + b, mu = a * b / p, oo2p = 0.5 / p, bp = b / p, ap = a / p;
            const double cc = sv.coefs[ka] * sv.coefs[kb];
            const double sq = sqpi / sqrt(p);
            double ex[LI + 1][LJ + 3][L + 3], ey[LI + 1][LJ + 3][L + 3], ez[LI + 1][LJ + 3][L + 3];
            hermite_e<LI, LJ + 2>(-bp * ABx, ap * ABx, oo2p, exp(-mu * ABx * ABx) * sq * cc, ex);
            hermite_e<LI, LJ + 2>(-bp * ABy, ap * ABy, oo2p, exp(-mu * ABy * ABy) * sq, ey);
            hermite_e<LI, LJ + 2>(-bp * ABz, ap * ABz, oo2p, exp(-mu * ABz * ABz) * sq, ez);
            const double Px = (a * Ax + b * Bx) / p - ox, Py = (a * Ay + b * By) / p - oy, Pz = (a * Az + b * Bz) / p - oz;
            // nuclear attraction: Rsum_h = sum_C (-Z_C 2 pi / p) R_h(p, P - C), P - C as A - C - (b/p)(A - B)
            double rsum[nherm(L)];
#pragma unroll
            for (int h = 0; h < nherm(L); ++h) rsum[h] = 0.0;
            for (int c = 0; c < sv.natm; ++c) {
                double R[nherm(L)];
                hermite_r<L>(p, (Ax - sv.pos[3 * c]) - bp * ABx, (Ay - sv.pos[3 * c + 1]) - bp * ABy,
                             (Az - sv.pos[3 * c + 2]) - bp * ABz, R);
                const double w = -sv.charges[c] * 2.0 * PI / p;
#pragma unroll
                for (int h = 0; h < nherm(L); ++h) rsum[h] += w * R[h];
            }
            const double e1 = 1.0 / (sq * sq * sq);   // V uses E without the sqrt(pi/p) factors
#pragma unroll
            for (int i = 0; i < NI; ++i) {
                const int ix = cart_x(LI, i), iy = cart_y(LI, i), iz = cart_z(LI, i);
#pragma unroll
                for (int j = 0; j < NJ; ++j) {
                    const int jx = cart_x(LJ, j), jy = cart_y(LJ, j), jz = cart_z(LJ, j);
                    const double sx = ex[ix][jx][0], sy = ey[iy][jy][0], sz = ez[iz][jz][0];
                    s[i][j] += sx * sy * sz;
                    t[i][j] += kin1d<LI, LJ + 2>(ex, ix, jx, b) * sy * sz + sx * kin1d<LI, LJ + 2>(ey, iy, jy, b) * sz +
                               sx * sy * kin1d<LI, LJ + 2>(ez, iz, jz, b);
                    mx[i][j] += (ex[ix][jx][1] + Px * sx) * sy * sz;
                    my[i][j] += sx * (ey[iy][jy][1] + Py * sy) * sz;
                    mz[i][j] += sx * sy * (ez[iz][jz][1] + Pz * sz);
                    double acc = 0.0;
#pragma unroll
                    for (int tt = 0; tt <= ix + jx; ++tt)
#pragma unroll
                        for (int uu = 0; uu <= iy + jy; ++uu)
#pragma unroll
                            for (int ww = 0; ww <= iz + jz; ++ww)
                                acc += ex[ix][jx][tt] * ey[iy][jy][uu] * ez[iz][jz][ww] * rsum[hidx(tt, uu, ww)];
                    vv[i][j] += acc * e1;
                }
            }
        }
    }
    const int n = sv.nao, oi = sv.ao[si], oj = sv.ao[sj];
    const size_t nn = (size_t)n * n;
#pragma unroll
    for (int i = 0; i < NI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const double f = cart_norm(cart_x(LI, i), cart_y(LI, i), cart_z(LI, i)) *
                             cart_norm(cart_x(LJ, j), cart_y(LJ, j), cart_z(LJ, j));
            const size_t a1 = (size_t)(oi + i) * n + oj + j, a2 = (size_t)(oj + j) * n + oi + i;
            S[a1] = f * s[i][j];
            T[a1] = f * t[i][j];
            M[a1] = f * mx[i][j];
            M[nn + a1] = f * my[i][j];
            M[2 * nn + a1] = f * mz[i][j];
            V[a1] = f * vv[i][j];
            if (si != sj) {     // a diagonal block holds both (i, j) and (j, i) already
                S[a2] = S[a1];
                T[a2] = T[a1];
                M[a2] = M[a1];
                M[nn + a2] = M[nn + a1];
                M[2 * nn + a2] = M[2 * nn + a1];
                V[a2] = V[a1];
            }
        }
}

// d/dR [ sum W S + sum D T ] (W with the sign the caller wants) and
// d/dR sum D V for shell pairs of class (LI, LJ); block-shared accumulator.
template <int LI, int LJ>
__global__ void __launch_bounds__(128) onee_grad_kernel(ShellView sv, int p_begin, int p_end,
                                                        const double* W, const double* Dm, facc* grad) {
    extern __shared__ facc gsh[];
    for (int i = threadIdx.x; i < 3 * sv.natm; i += blockDim.x) gsh[i] = 0;
    __syncthreads();
    const int ip = p_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (ip < p_end) {
        const int si = sv.pair_i[ip], sj = sv.pair_j[ip];
        constexpr int NI = ncart(LI), NJ = ncart(LJ), L = LI + LJ;
        const int ai = sv.atom[si], aj = sv.atom[sj];
        const int n = sv.nao, oi = sv.ao[si], oj = sv.ao[sj];
        const double Ax = sv.pos[3 * ai], Ay = sv.pos[3 * ai + 1], Az = sv.pos[3 * ai + 2];
        const double ABx = Ax - sv.pos[3 * aj], ABy = Ay - sv.pos[3 * aj + 1], ABz = Az - sv.pos[3 * aj + 2];
        const double sym = si != sj ? 2.0 : 1.0;
        double wv[NI][NJ], dv[NI][NJ];
#pragma unroll
        for (int i = 0; i < NI; ++i)
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const double f = cart_norm(cart_x(LI, i), cart_y(LI, i), cart_z(LI, i)) *
                                 cart_norm(cart_x(LJ, j), cart_y(LJ, j), cart_z(LJ, j));
                wv[i][j] = f * W[(size_t)(oi + i) * n + oj + j];
                dv[i][j] = f * Dm[(size_t)(oi + i) * n + oj + j];
            }
        double gA[3] = {0.0, 0.0, 0.0};      // overlap + kinetic, centre A (B gets -gA)
        double gNA[3] = {0.0, 0.0, 0.0};     // nuclear attraction, centre A
        double gNB[3] = {0.0, 0.0, 0.0};     // nuclear attraction, centre B
        const double sqpi = sqrt(PI);
        for (int ka = sv.p0[si]; ka < sv.p0[si] + sv.np[si]; ++ka) {
            const double a = sv.exps[ka];
            for (int kb = sv.p0[sj]; kb < sv.p0[sj] + sv.np[sj]; ++kb) {
                const double b = sv.exps[kb], p = a + b, mu = a * b / p, oo2p = 0.5 / p, bp = b / p, ap = a / p;
                const double cc = sv.coefs[ka] * sv.coefs[kb];
                const double sq = sqpi / sqrt(p);
                double ex[LI + 2][LJ + 3][L + 4], ey[LI + 2][LJ + 3][L + 4], ez[LI + 2][LJ + 3][L + 4];
                hermite_e<LI + 1, LJ + 2>(-bp * ABx, ap * ABx, oo2p, exp(-mu * ABx * ABx) * sq * cc, ex);
                hermite_e<LI + 1, LJ + 2>(-bp * ABy, ap * ABy, oo2p, exp(-mu * ABy * ABy) * sq, ey);
                hermite_e<LI + 1, LJ + 2>(-bp * ABz, ap * ABz, oo2p, exp(-mu * ABz * ABz) * sq, ez);
                // overlap and kinetic (only between different atoms; pairs si > sj)
                if (ai != aj) {
#pragma unroll
                    for (int i = 0; i < NI; ++i)
#pragma unroll
                        for (int j = 0; j < NJ; ++j) {
                            const int I3[3] = {cart_x(LI, i), cart_y(LI, i), cart_z(LI, i)};
                            const int J3[3] = {cart_x(LJ, j), cart_y(LJ, j), cart_z(LJ, j)};
                            double S1[3], K1[3], dS[3], dK[3];
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                const auto& e = d == 0 ? ex : (d == 1 ? ey : ez);
                                const int ii = I3[d], jj = J3[d];
                                S1[d] = e[ii][jj][0];
                                K1[d] = kin1d<LI + 1, LJ + 2>(e, ii, jj, b);
                                dS[d] = 2.0 * a * e[ii + 1][jj][0];
                                dK[d] = 2.0 * a * kin1d<LI + 1, LJ + 2>(e, ii + 1, jj, b);
                                if (ii > 0) {
                                    dS[d] -= ii * e[ii - 1][jj][0];
                                    dK[d] -= ii * kin1d<LI + 1, LJ + 2>(e, ii - 1, jj, b);
                                }
                            }
                            const double w2 = 2.0 * wv[i][j], d2 = 2.0 * dv[i][j];
                            gA[0] += w2 * dS[0] * S1[1] * S1[2] + d2 * (dK[0] * S1[1] * S1[2] + dS[0] * (K1[1] * S1[2] + S1[1] * K1[2]));
                            gA[1] += w2 * S1[0] * dS[1] * S1[2] + d2 * (dK[1] * S1[0] * S1[2] + dS[1] * (K1[0] * S1[2] + S1[0] * K1[2]));
                            gA[2] += w2 * S1[0] * S1[1] * dS[2] + d2 * (dK[2] * S1[0] * S1[1] + dS[2] * (K1[0] * S1[1] + S1[0] * K1[1]));
                        }
                }
                // nuclear attraction: density-contracted Hermite vectors of the pair and of d/dA
                constexpr int NH0 = nherm(L), NH1 = nherm(L + 1);
                double dE[NH0], dA[3][NH1];
#pragma unroll
                for (int h = 0; h < NH0; ++h) dE[h] = 0.0;
#pragma unroll
                for (int h = 0; h < NH1; ++h) dA[0][h] = dA[1][h] = dA[2][h] = 0.0;
                const double e1 = 1.0 / (sq * sq * sq);
#pragma unroll
                for (int i = 0; i < NI; ++i)
#pragma unroll
                    for (int j = 0; j < NJ; ++j) {
                        const int ix = cart_x(LI, i), iy = cart_y(LI, i), iz = cart_z(LI, i);
                        const int jx = cart_x(LJ, j), jy = cart_y(LJ, j), jz = cart_z(LJ, j);
                        const double w = sym * dv[i][j] * e1;
#pragma unroll
                        for (int tt = 0; tt <= ix + jx + 1; ++tt)
#pragma unroll
                            for (int uu = 0; uu <= iy + jy + 1; ++uu)
#pragma unroll
                                for (int ww = 0; ww <= iz + jz + 1; ++ww) {
                                    const double exv = ex[ix][jx][tt], eyv = ey[iy][jy][uu], ezv = ez[iz][jz][ww];
                                    double dxv = 2.0 * a * ex[ix + 1][jx][tt], dyv = 2.0 * a * ey[iy + 1][jy][uu],
                                           dzv = 2.0 * a * ez[iz + 1][jz][ww];
                                    if (ix > 0) dxv -= ix * ex[ix - 1][jx][tt];
                                    if (iy > 0) dyv -= iy * ey[iy - 1][jy][uu];
                                    if (iz > 0) dzv -= iz * ez[iz - 1][jz][ww];
                                    const int h = hidx(tt, uu, ww);
                                    if (tt <= ix + jx && uu <= iy + jy && ww <= iz + jz) dE[h] += w * exv * eyv * ezv;
                                    if (tt + uu + ww <= L + 1) {
                                        dA[0][h] += w * dxv * eyv * ezv;
                                        dA[1][h] += w * exv * dyv * ezv;
                                        dA[2][h] += w * exv * eyv * dzv;
                                    }
                                }
                    }
                for (int c = 0; c < sv.natm; ++c) {
                    double R[NH1];
                    hermite_r<L + 1>(p, (Ax - sv.pos[3 * c]) - bp * ABx, (Ay - sv.pos[3 * c + 1]) - bp * ABy,
                                     (Az - sv.pos[3 * c + 2]) - bp * ABz, R);
                    const double pref = -sv.charges[c] * 2.0 * PI / p;
                    double ga[3] = {0.0, 0.0, 0.0}, gc[3] = {0.0, 0.0, 0.0};
#pragma unroll
                    for (int h = 0; h < NH1; ++h) {
                        ga[0] += dA[0][h] * R[h];
                        ga[1] += dA[1][h] * R[h];
                        ga[2] += dA[2][h] * R[h];
                    }
#pragma unroll
                    for (int tt = 0; tt <= L; ++tt)
#pragma unroll
                        for (int uu = 0; uu <= L - tt; ++uu)
#pragma unroll
                            for (int ww = 0; ww <= L - tt - uu; ++ww) {
                                const double de = dE[hidx(tt, uu, ww)];
                                gc[0] -= de * R[hidx(tt + 1, uu, ww)];
                                gc[1] -= de * R[hidx(tt, uu + 1, ww)];
                                gc[2] -= de * R[hidx(tt, uu, ww + 1)];
                            }
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        ga[d] *= pref;
                        gc[d] *= pref;
                        gNA[d] += ga[d];
                        gNB[d] -= ga[d] + gc[d];
                        fadd(&gsh[3 * c + d], gc[d], FIX_G);
                    }
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            fadd(&gsh[3 * ai + d], gA[d] + gNA[d], FIX_G);
            fadd(&gsh[3 * aj + d], -gA[d] + gNB[d], FIX_G);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * sv.natm; i += blockDim.x)
        if (gsh[i] != 0) atomicAdd(&grad[i], gsh[i]);
}

}  // namespace hf
