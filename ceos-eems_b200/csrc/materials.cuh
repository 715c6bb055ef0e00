// materials.cuh -- Gauss-point constitutive updates on the device.
//
// Each model maps the deformation gradient F (and the committed state) to the Cauchy stress
// (Voigt, 6), the spatial tangent D (upper triangle, 21 packed entries, read as symmetric the
// way the reference's dsymm 'L','U' reads it, ModMathRoutines.f90:975-1000) and the new state.
// T is the element arithmetic type (double for CEOS_FP64, float for CEOS_MIXED); det F and
// ln J are always formed in FP64, as is the J2 return-mapping scalar.
#pragma once
#include "ceos_common.cuh"

namespace ceos {

enum : int { M_J2_SMALL = 2, M_NH_Q1P0 = 4, M_SVK = 5, M_CNH = 7, M_VISCO_VAR = 12, M_VISCO_PRONY = 101, M_J2_FINITE = 102,
             M_EXTERNAL = 200 };

template <int MODEL>
struct ModelInfo;
template <>
struct ModelInfo<M_CNH> { static constexpr int nstate = 0, nparams = 2; };
template <>
struct ModelInfo<M_SVK> { static constexpr int nstate = 0, nparams = 2; };
template <>
struct ModelInfo<M_NH_Q1P0> { static constexpr int nstate = 0, nparams = 2; };
template <>
struct ModelInfo<M_J2_SMALL> { static constexpr int nstate = 7, nparams = 4; };
template <>
struct ModelInfo<M_VISCO_PRONY> { static constexpr int nstate = 30, nparams = 11; };
template <>
struct ModelInfo<M_J2_FINITE> { static constexpr int nstate = 7, nparams = 4; };
template <>
struct ModelInfo<M_VISCO_VAR> { static constexpr int nstate = 19, nparams = 6; };
// External constitutive response: the "state" of each Gauss point holds its Cauchy stress (6)
// and spatial tangent (21 upper entries), written by another kernel before the element loop
// (the learned FE^2 surrogate, or RVE solves); one unused parameter.
template <>
struct ModelInfo<M_EXTERNAL> { static constexpr int nstate = 27, nparams = 1; };

// ---------------------------------------------------------------------------------------
// Compressible Neo-Hookean (ConstitutiveModelsLibrary/ModCompressibleNeoHookean.f90:422-546):
//   sigma = Mu/J (b - I) + Lambda/J ln J I;  D = Lambda/J I(x)I + 2/J (Mu - Lambda ln J) Isym.
// ---------------------------------------------------------------------------------------
template <typename T>
CEOS_D void cnh_update(const T F[3][3], const T* p, T sig[6], T D[21]) {
    const T Mu = p[0], Lambda = p[1];
    T b[6];
    ffT(F, b);
    const double Jd = det3_fp64(F);
    const T J = (T)Jd;
    const T lnJ = (T)log(Jd);
    const T a = Mu / J, c = (Lambda / J) * lnJ;
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = a * (b[k] - (T)delta6(k)) + (T)delta6(k) * c;
    const T l = Lambda / J, m = (T(2) / J) * (Mu - Lambda * lnJ);
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 6; ++j) D[up21(i, j)] = l * (T)(delta6(i) * delta6(j)) + (i == j ? (i < 3 ? m : T(0.5) * m) : T(0));
}

// ---------------------------------------------------------------------------------------
// Neo-Hookean of the Mean Dilatation element (ConstitutiveModelsLibrary/ModNeoHookeanQ1P0.f90):
//   sigma = 2 C10 J^(-5/3) (b - tr(b)/3 I) + pbar I,  pbar = 3 K (Jbar^(1/3) - 1) / Jbar^(2/3)
// (:429-484); tangent = push-forward of C_iso + C_p with C = F^T F (:540-613):
//   C_iso = 2/3 J^(-2/3) (Sf:C) P - 2/3 (S_iso (x) C^-1 + C^-1 (x) S_iso),
//   P = C^-1 [.] C^-1 - 1/3 C^-1 (x) C^-1,  C_p = J pbar (C^-1 (x) C^-1 - 2 C^-1 [.] C^-1),
// with Sf = 2 C10 I, S_iso = J^(-2/3) (Sf - 1/3 (Sf:C) C^-1), [.] the minor-symmetric product
// 1/4 (A_ik B_jl + A_il B_jk + A_jk B_il + A_jl B_ik) (Square_Voigt, ModMathRoutines.f90:581-625),
// and the push-forward Q W Q^T / J (Push_Forward_Voigt, :254-311).  params [C10, BulkModulus];
// Jbar = V / V0 of the element (SubSolveConstitutiveModel.f90:100).  Scalars in FP64.
// ---------------------------------------------------------------------------------------
template <typename T>
CEOS_D T sym_at(const T v[6], int i, int j) {  // entry (i, j) of a symmetric tensor in Voigt
    return i == j ? v[i] : v[(i + j == 1) ? 3 : ((i + j == 3) ? 4 : 5)];
}
template <typename T>
CEOS_D void nh_q1p0_update(const T F[3][3], const T* p, double Jbar, T sig[6], T D[21]) {
    const double C10 = p[0], K = p[1];
    T b[6], Cv[6];
    ffT(F, b);
    fTf(F, Cv);
    const double J = det3_fp64(F);
    const double jb13 = cbrt(Jbar);
    const double pbar = 3.0 * K * (jb13 - 1.0) / (jb13 * jb13);
    const double Jm23 = 1.0 / cbrt(J * J), Jm53 = Jm23 / J;
    const T trb = b[0] + b[1] + b[2];
#pragma unroll
    for (int k = 0; k < 6; ++k)
        sig[k] = (T)(2.0 * C10 * Jm53) * (b[k] - (k < 3 ? trb / T(3) : T(0))) + (k < 3 ? (T)pbar : T(0));
    // C^-1 (Voigt) by the adjugate
    T Cm[3][3], Ci[3][3];
    sym_to_mat(Cv, Cm);
    inv3(Cm, det3(Cm), Ci);
    const T civ[6] = {Ci[0][0], Ci[1][1], Ci[2][2], Ci[0][1], Ci[1][2], Ci[0][2]};
    const T sc = T(2.0 * C10) * (Cv[0] + Cv[1] + Cv[2]);  // Sf : C
    T siso[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) siso[k] = (T)Jm23 * ((k < 3 ? T(2.0 * C10) : T(0)) - sc / T(3) * civ[k]);
    const int vi[6] = {0, 1, 2, 0, 1, 0}, vj[6] = {0, 1, 2, 1, 2, 2};
    T Cb[6][6];
#pragma unroll
    for (int pp = 0; pp < 6; ++pp)
#pragma unroll
        for (int qq = 0; qq < 6; ++qq) {
            const int i = vi[pp], j = vj[pp], k = vi[qq], l = vj[qq];
            const T sq = T(0.25) * (sym_at(civ, i, k) * sym_at(civ, j, l) + sym_at(civ, i, l) * sym_at(civ, j, k) +
                                    sym_at(civ, j, k) * sym_at(civ, i, l) + sym_at(civ, j, l) * sym_at(civ, i, k));
            const T bl = civ[pp] * civ[qq];
            const T ciso = T(2.0 / 3.0) * (T)Jm23 * sc * (sq - bl / T(3)) -
                           T(2.0 / 3.0) * (siso[pp] * civ[qq] + civ[pp] * siso[qq]);
            const T cp = (T)(J * pbar) * (bl - T(2) * sq);
            Cb[pp][qq] = ciso + cp;
        }
    // push-forward: Q Cb Q^T / J, Q[p][r] = F_iI F_jJ (+ F_iJ F_jI for shear r)
    T Q[6][6];
#pragma unroll
    for (int pp = 0; pp < 6; ++pp)
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            const int i = vi[pp], j = vj[pp], I = vi[r], Jx = vj[r];
            Q[pp][r] = F[i][I] * F[j][Jx] + (r >= 3 ? F[i][Jx] * F[j][I] : T(0));
        }
    T QC[6][6];
#pragma unroll
    for (int pp = 0; pp < 6; ++pp)
#pragma unroll
        for (int qq = 0; qq < 6; ++qq) {
            T t = 0;
#pragma unroll
            for (int r = 0; r < 6; ++r) t += Q[pp][r] * Cb[r][qq];
            QC[pp][qq] = t;
        }
    const T rJ = (T)(1.0 / J);
#pragma unroll
    for (int pp = 0; pp < 6; ++pp)
#pragma unroll
        for (int qq = pp; qq < 6; ++qq) {
            T t = 0;
#pragma unroll
            for (int r = 0; r < 6; ++r) t += QC[pp][r] * Q[qq][r];
            D[up21(pp, qq)] = t * rJ;
        }
}
// SecondDerivativesOfPSI_Jbar_NeoHookeanQ1P0 (ModNeoHookeanQ1P0.f90:625-652)
CEOS_D double nh_q1p0_d2psi(double K, double Jbar) {
    const double jb13 = cbrt(Jbar);
    return -(K * (jb13 - 2.0)) / (Jbar * jb13 * jb13);
}

// ---------------------------------------------------------------------------------------
// St Venant-Kirchhoff (ModStVenantKirchhoff.f90:643-780): S = Lambda trE I + 2 Mu E,
// sigma = F S F^T / J, c_ijkl = Lambda/J b_ij b_kl + Mu/J (b_ik b_jl + b_il b_jk).
// params [YoungModulus, Poisson] -> Lambda, Mu as (:238-239).
// ---------------------------------------------------------------------------------------
template <typename T>
CEOS_D void svk_update(const T F[3][3], const T* p, T sig[6], T D[21]) {
    const T E = p[0], nu = p[1];
    const T Lambda = nu * E / ((T(1) + nu) * (T(1) - T(2) * nu));
    const T Mu = E / (T(2) * (T(1) + nu));
    T C[6], S[6], b[6];
    fTf(F, C);
    T Eg[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) Eg[k] = T(0.5) * (C[k] - (T)delta6(k));
    const T trE = Eg[0] + Eg[1] + Eg[2];
#pragma unroll
    for (int k = 0; k < 6; ++k) S[k] = Lambda * trE * (T)delta6(k) + T(2) * Mu * Eg[k];
    const T J = (T)det3_fp64(F);
    T tau[6];
    push_sym(F, S, tau);
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = tau[k] / J;
    ffT(F, b);
    T bm[3][3];
    sym_to_mat(b, bm);
    const int I[6] = {0, 1, 2, 0, 1, 0}, Jx[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int c = a; c < 6; ++c) {
            const int i = I[a], j = Jx[a], k = I[c], l = Jx[c];
            D[up21(a, c)] = (Lambda / J) * bm[i][j] * bm[k][l] + (Mu / J) * (bm[i][k] * bm[j][l] + bm[i][l] * bm[j][k]);
        }
}

// ---------------------------------------------------------------------------------------
// J2 plasticity, small strain, as the reference implements it (ModJ2Plasticity.f90:385-479
// update, :555-620 tangent).  strain = (F11-1, F22-1, F33-1, F12+F21, F23+F32, F13+F31);
// state = [plastic strain (6), accumulated plastic strain].
// ---------------------------------------------------------------------------------------
template <typename T>
CEOS_D void j2_small_update(const T F[3][3], const T* p, const T* st, T* stn, T sig[6], T D[21]) {
    const T E = p[0], nu = p[1], sy = p[2], H = p[3];
    T Strain[6] = {F[0][0] - T(1), F[1][1] - T(1), F[2][2] - T(1), F[0][1] + F[1][0], F[1][2] + F[2][1],
                   F[0][2] + F[2][0]};
    const T K = E / (T(3) * (T(1) - T(2) * nu));
    const T G = E / (T(2) * (T(1) + nu));
    T Ee[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) Ee[k] = Strain[k] - st[k];
    const T Evol = Ee[0] + Ee[1] + Ee[2];
    T Sd[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) Sd[k] = G * (Ee[k] - Evol * (T)delta6(k) / T(3)) * (k < 3 ? T(2) : T(1));
    const T p_t = K * Evol;
    const double q = sqrt(1.5 * ((double)Sd[0] * Sd[0] + (double)Sd[1] * Sd[1] + (double)Sd[2] * Sd[2] +
                                 2.0 * Sd[3] * Sd[3] + 2.0 * Sd[4] * Sd[4] + 2.0 * Sd[5] * Sd[5]));
    const double phi = q - ((double)sy + (double)H * st[6]);
    if (phi <= 0.0) {
#pragma unroll
        for (int k = 0; k < 7; ++k) stn[k] = st[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) sig[k] = Sd[k] + p_t * (T)delta6(k);
        const T cte = E / ((T(1) + nu) * (T(1) - T(2) * nu));
#pragma unroll
        for (int i = 0; i < 21; ++i) D[i] = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j) D[up21(i, j)] = cte * (i == j ? T(1) - nu : nu);
#pragma unroll
        for (int i = 3; i < 6; ++i) D[up21(i, i)] = cte * (T(0.5) - nu);
    } else {
        const double dgam = phi / (3.0 * (double)G + (double)H);
        const T r = (T)(1.0 - dgam * 3.0 * (double)G / q);
        T S[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            S[k] = r * Sd[k];
            sig[k] = S[k] + p_t * (T)delta6(k);
            stn[k] = Strain[k] - (S[k] / (T(2) * G) + Evol * (T)delta6(k) / T(3));
        }
        stn[6] = (T)((double)st[6] + dgam);
        const T nrm = (T)(q / sqrt(1.5));
        T N[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) N[k] = Sd[k] / nrm;
        const T c1 = T(2) * G * r;
        const T c2 = (T)(6.0 * (double)G * G * (dgam / q - 1.0 / (3.0 * (double)G + (double)H)));
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j) {
                const T Id = (i == j ? (i < 3 ? T(1) : T(0.5)) : T(0)) - (T)(delta6(i) * delta6(j)) / T(3);
                D[up21(i, j)] = c1 * Id + c2 * N[i] * N[j] + K * (T)(delta6(i) * delta6(j));
            }
    }
}

// ---------------------------------------------------------------------------------------
// Finite-strain generalized Maxwell (project-defined): decoupled Neo-Hookean ground state
// Psi = K/2 (ln J)^2 + mu/2 (I1bar - 3) and nb <= 4 Maxwell branches on the isochoric stress,
// recursive update of Holzapfel, Nonlinear Solid Mechanics (2000) 6.10 (after Simo 1987):
//   Q_a^{n+1} = e_a (e_a Q_a^n - beta_a S_iso^n) + beta_a e_a S_iso^{n+1},  e_a = exp(-dt/(2 tau_a));
//   c = c_vol + (1 + sum beta_a e_a) c_iso.
// params [mu, K, nb, beta1, tau1, ..., beta4, tau4]; state [S_iso^n (6), Q_1..Q_4 (6 each)].
// ---------------------------------------------------------------------------------------
template <typename T, typename IO>
CEOS_D void visco_prony_update(const T F[3][3], const T* p, const T* ebr, const IO& io, T sig[6], T D[21]) {
    // ebr[a] = exp(-dt / (2 tau_a)) for the branches (computed once per launch)
    const T mu = p[0], K = p[1];
    const int nb = (int)p[2];
    T C[6];
    fTf(F, C);
    const double Jd = det3_fp64(F);
    const double lnJd = log(Jd);
    const T J = (T)Jd, lnJ = (T)lnJd;
    const T J23 = texp<T>(T(-2.0 / 3.0) * lnJ);
    T Siso[6];
    {
        T Ci[6];
        inv_sym(C, (T)(Jd * Jd), Ci);
        const T trC3 = (C[0] + C[1] + C[2]) * T(1.0 / 3.0);
        const T muJ = mu * J23;
#pragma unroll
        for (int k = 0; k < 6; ++k) Siso[k] = muJ * ((T)delta6(k) - trC3 * Ci[k]);
    }
    T Qs[6] = {0, 0, 0, 0, 0, 0};
    T dsum = T(0);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        if (a < nb) {
            const T beta = p[3 + 2 * a];
            const T e = ebr[a];
            const T be = beta * e;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const T q = e * (e * io.ld(6 + 6 * a + k) - beta * io.ld(k)) + be * Siso[k];
                io.st(6 + 6 * a + k, q);
                Qs[k] += q;
            }
            dsum += be;
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) io.st(k, Siso[k]);
    T tq[6];
    push_sym(F, Qs, tq);
    T b[6];
    ffT(F, b);
    const T trb = b[0] + b[1] + b[2];
    T tiso[6];
    const T invJ = T(1) / J;
    const T pv = K * lnJ * invJ;
    const T muJ = mu * J23;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        tiso[k] = muJ * (b[k] - trb * T(1.0 / 3.0) * (T)delta6(k));
        sig[k] = pv * (T)delta6(k) + (tiso[k] + tq[k]) * invJ;
    }
    const T I1b = J23 * trb;
    const T f = (T(1) + dsum) * invJ;
    const T kj = K * invJ;
    const T c23 = T(2.0 / 3.0) * mu * I1b;
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int c = a; c < 6; ++c) {
            const T Is = (a == c ? (a < 3 ? T(1) : T(0.5)) : T(0));
            const T dd = (T)(delta6(a) * delta6(c));
            const T vol = kj * dd - T(2) * pv * Is;
            const T iso = c23 * (Is - dd * T(1.0 / 3.0)) - T(2.0 / 3.0) * (tiso[a] * (T)delta6(c) + (T)delta6(a) * tiso[c]);
            D[up21(a, c)] = vol + f * iso;
        }
}

// ---------------------------------------------------------------------------------------
// Multiplicative finite-strain J2 (project-defined): Simo (1988), Simo & Hughes (1998) Box 9.1.
// Trial b_e = F Cp^{-1} F^T, s = mu dev(bbar_e), radial return with linear isotropic hardening
// (closed form, FP64), U(J) = K/2 (1/2 (J^2 - 1) - ln J).  Tangent from the Lie derivative of
// tau, symmetrized.  params [E, nu, sigma_y0, H]; state [Cp^{-1} (Voigt 6), alpha].
// ---------------------------------------------------------------------------------------
template <typename T>
CEOS_D void j2_finite_update(const T F[3][3], const T* p, const T* st, T* stn, T sig[6], T D[21]) {
    const T E = p[0], nu = p[1];
    const double sy = p[2], H = p[3];
    const T mu = E / (T(2) * (T(1) + nu));
    const T K = E / (T(3) * (T(1) - T(2) * nu));
    T be[6];
    push_sym(F, st, be);  // F Cp^{-1} F^T
    const double Jd = det3_fp64(F);
    const double lnJd = log(Jd);
    const T J = (T)Jd;
    // J^(-2/3) from the FP64 ln J; the power itself in the element arithmetic type
    const T J23 = texp<T>((T)(-2.0 / 3.0 * lnJd));
    const T Ie = J23 * (be[0] + be[1] + be[2]) / T(3);
    const T mub = mu * Ie;
    T s[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = mu * (J23 * be[k] - Ie * (T)delta6(k));
    const double nsd = sqrt((double)s[0] * s[0] + (double)s[1] * s[1] + (double)s[2] * s[2] +
                            2.0 * ((double)s[3] * s[3] + (double)s[4] * s[4] + (double)s[5] * s[5]));
    const double alpha = st[6];
    const double fd = nsd - sqrt(2.0 / 3.0) * (sy + H * alpha);
    const bool plastic = fd > 0.0;
    const double inv_h = 1.0 / (3.0 * (double)mub + H);
    T n[6];
    const T ns = (T)nsd;
#pragma unroll
    for (int k = 0; k < 6; ++k) n[k] = nsd > 0.0 ? s[k] / ns : T(0);
    double gd = 0.0;
    T snew[6];
    if (plastic) {
        // gd = 3 mub fd / (3 mub + H); the alpha increment sqrt(2/3) gd / (2 mub) = sqrt(2/3) 1.5 fd / (3 mub + H)
        gd = 3.0 * (double)mub * fd * inv_h;
        stn[6] = (T)(alpha + sqrt(2.0 / 3.0) * 1.5 * fd * inv_h);
    } else {
        stn[6] = (T)alpha;
    }
    const T g = (T)gd;
#pragma unroll
    for (int k = 0; k < 6; ++k) snew[k] = s[k] - g * n[k];
    // Cp^{-1} = J^{2/3} F^{-1} (s/mu + Ie I) F^{-T}
    {
        T Fi[3][3];
        inv3(F, J, Fi);
        T bb[6];
        const T Jp23 = T(1) / J23;
#pragma unroll
        for (int k = 0; k < 6; ++k) bb[k] = (snew[k] / mu + Ie * (T)delta6(k)) * Jp23;
        push_sym(Fi, bb, stn);
    }
    const T Jp = T(0.5) * K * (J * J - T(1));
    const T invJ = T(1) / J;
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = (Jp * (T)delta6(k) + snew[k]) * invJ;
    // tangent
    T n2[6];
    {
        T nm[3][3];
        sym_to_mat(n, nm);
        const int I[6] = {0, 1, 2, 0, 1, 0}, Jx[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
        for (int k = 0; k < 6; ++k) n2[k] = nm[I[k]][0] * nm[0][Jx[k]] + nm[I[k]][1] * nm[1][Jx[k]] + nm[I[k]][2] * nm[2][Jx[k]];
    }
    const T beta1 = plastic ? (T)(gd / nsd) : T(0);
    const T b0inv = plastic ? (T)(3.0 * (double)mub * inv_h) : T(0);
    const T cH = plastic ? (T)(2.0 * fd * H * nsd * inv_h * inv_h) : T(0);
    const T KJ2 = K * J * J, KJ21 = K * (J * J - T(1));
    const T w1 = b0inv - beta1;
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int c = a; c < 6; ++c) {
            const T Isac = (a == c ? (a < 3 ? T(1) : T(0.5)) : T(0));
            const T dd = (T)(delta6(a) * delta6(c));
            const T dev = T(2) * mub * (Isac - dd / T(3)) - T(2.0 / 3.0) * (s[a] * (T)delta6(c) + (T)delta6(a) * s[c]);
            T Aac = dev, Aca = dev;
            if (plastic) {
                const T vc = T(2) * mub * n[c] - T(2.0 / 3.0) * ns * (T)delta6(c) + T(2) * ns * n2[c];
                const T va = T(2) * mub * n[a] - T(2.0 / 3.0) * ns * (T)delta6(a) + T(2) * ns * n2[a];
                Aac = (T(1) - beta1) * dev - n[a] * (w1 * vc + cH * n[c]);
                Aca = (T(1) - beta1) * dev - n[c] * (w1 * va + cH * n[a]);
            }
            D[up21(a, c)] = (KJ2 * dd - KJ21 * Isac + T(0.5) * (Aac + Aca)) * invJ;
        }
}

}  // namespace ceos
