// ceos_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the parity checker, never the product).
//
// FP64 CPU restatement of the CEOS element loop of one Newton iteration and of the host
// driver around it.  Every routine cites the reference file:line it restates (paths are
// relative to the reference's SourceCode/ folder).  The product library (ceos-eems_b200)
// never includes, links or calls this file.
#include "ceos_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------------------
// Hexa8 (FEM/Elements/ElementLibrary/ModElementHexa8.f90:150-329)
// ---------------------------------------------------------------------------------------
const double kNodeSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// GetDifShapeFunctions_Hexa8 (:211-268): dN(i, d) at natural coordinates xi.
void hexa8_dN(const double xi[3], double dN[8][3]) {
    for (int i = 0; i < 8; ++i)
        dN[i][0] = kNodeSign[i][0] * (1.0 + kNodeSign[i][1] * xi[1]) * (1.0 + kNodeSign[i][2] * xi[2]) / 8.0;
    for (int i = 0; i < 8; ++i)
        dN[i][1] = kNodeSign[i][1] * (1.0 + kNodeSign[i][0] * xi[0]) * (1.0 + kNodeSign[i][2] * xi[2]) / 8.0;
    for (int i = 0; i < 8; ++i)
        dN[i][2] = kNodeSign[i][2] * (1.0 + kNodeSign[i][0] * xi[0]) * (1.0 + kNodeSign[i][1] * xi[1]) / 8.0;
}

// AllocateGaussPointsParameters_Hexa8 (:278-329): 2x2x2 points at +-1/sqrt(3), weight 1.
void hexa8_gp(int gp, double xi[3], double* w) {
    const double x = 1.0 / std::sqrt(3.0);
    for (int d = 0; d < 3; ++d) xi[d] = kNodeSign[gp][d] * x;
    *w = 1.0;
}

// ---------------------------------------------------------------------------------------
// Small dense helpers (Tools/MathTools/ModMathRoutines.f90:16-62)
// ---------------------------------------------------------------------------------------
typedef double M3[3][3];

double det3(const M3 M) {  // det (:16-31), same term order
    return M[0][0] * M[1][1] * M[2][2] + M[0][1] * M[1][2] * M[2][0] + M[0][2] * M[1][0] * M[2][1] -
           M[0][2] * M[1][1] * M[2][0] - M[0][1] * M[1][0] * M[2][2] - M[0][0] * M[1][2] * M[2][1];
}

void inv3(const M3 A, M3 B) {  // inverse (:33-62), adjugate / det
    const double d = det3(A);
    B[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    B[0][1] = A[0][2] * A[2][1] - A[0][1] * A[2][2];
    B[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
    B[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    B[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
    B[1][2] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
    B[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    B[2][1] = A[0][1] * A[2][0] - A[0][0] * A[2][1];
    B[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] /= d;
}

void matmul3(const M3 A, const M3 B, M3 C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A[i][k] * B[k][j];
            C[i][j] = s;
        }
}
void transpose3(const M3 A, M3 B) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] = A[j][i];
}
// Convert_to_Voigt_3D_Sym (ModMathRoutines.f90:660-674): 11,22,33,12,23,13
void to_voigt(const M3 A, double v[6]) {
    v[0] = A[0][0]; v[1] = A[1][1]; v[2] = A[2][2];
    v[3] = A[0][1]; v[4] = A[1][2]; v[5] = A[0][2];
}
void from_voigt(const double v[6], M3 A) {
    A[0][0] = v[0]; A[1][1] = v[1]; A[2][2] = v[2];
    A[0][1] = A[1][0] = v[3];
    A[1][2] = A[2][1] = v[4];
    A[0][2] = A[2][0] = v[5];
}
const int kVi[6] = {0, 1, 2, 0, 1, 0};
const int kVj[6] = {0, 1, 2, 1, 2, 2};
const double kDelta[6] = {1, 1, 1, 0, 0, 0};
const double kIsym[6] = {1, 1, 1, 0.5, 0.5, 0.5};  // IsymV (ModMathRoutines.f90:194-207)

// StressTransformation second Piola -> Cauchy (Tools/ModContinuumMechanics.f90:152-162)
void pk2_to_cauchy(const M3 F, const M3 S, M3 sig) {
    const double J = det3(F);
    M3 Ft, T, T2;
    transpose3(F, Ft);
    matmul3(S, Ft, T);
    matmul3(F, T, T2);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sig[i][j] = (1.0 / J) * T2[i][j];
}

// ---------------------------------------------------------------------------------------
// Material models
// ---------------------------------------------------------------------------------------

// Compressible Neo-Hookean, UpdateStressAndStateVariables_CompressibleNeoHookean_3D
// (ConstitutiveModelsLibrary/ModCompressibleNeoHookean.f90:422-482) and
// GetTangentModulus_CompressibleNeoHookean_3D (:493-546).  params = [Mu, Lambda].
void cnh(const double* p, const M3 F, double sig[6], double D[36]) {
    const double Mu = p[0], Lambda = p[1];
    M3 Ft, b, S;
    transpose3(F, Ft);
    matmul3(F, Ft, b);
    const double J = det3(F);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            S[i][j] = (Mu / J) * (b[i][j] - (i == j ? 1.0 : 0.0)) +
                      (Lambda / J) * std::log(J) * (i == j ? 1.0 : 0.0);
    to_voigt(S, sig);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
            D[i * 6 + j] = (Lambda / J) * kDelta[i] * kDelta[j] +
                           (2.0 / J) * (Mu - Lambda * std::log(J)) * (i == j ? kIsym[i] : 0.0);
}

// Voigt products of ModMathRoutines.f90 (tensor components, order 11,22,33,12,23,13):
// Ball_Voigt (:532-577) A (x) B; Square_Voigt (:581-625), the minor-symmetric
// 1/4 (A_ik B_jl + A_il B_jk + A_jk B_il + A_jl B_ik); Inner_Product_Voigt (:629-638).
// (kVi, kVj: the Voigt index pairs above)
double vget(const double a[6], int i, int j) {  // symmetric tensor entry from Voigt
    for (int p = 0; p < 6; ++p)
        if ((kVi[p] == i && kVj[p] == j) || (kVi[p] == j && kVj[p] == i)) return a[p];
    return 0.0;
}
void ball_voigt(const double A[6], const double B[6], double T[36]) {
    for (int p = 0; p < 6; ++p)
        for (int q = 0; q < 6; ++q) T[p * 6 + q] = A[p] * B[q];
}
void square_voigt(const double A[6], const double B[6], double T[36]) {
    for (int p = 0; p < 6; ++p)
        for (int q = 0; q < 6; ++q) {
            const int i = kVi[p], j = kVj[p], k = kVi[q], l = kVj[q];
            T[p * 6 + q] = 0.25 * (vget(A, i, k) * vget(B, j, l) + vget(A, i, l) * vget(B, j, k) +
                                   vget(A, j, k) * vget(B, i, l) + vget(A, j, l) * vget(B, i, k));
        }
}
double inner_voigt(const double A[6], const double B[6]) {
    return A[0] * B[0] + A[1] * B[1] + A[2] * B[2] + 2.0 * (A[3] * B[3] + A[4] * B[4] + A[5] * B[5]);
}
// Push_Forward_Voigt (:254-311): T = A W A^T / J, A the Voigt map of F (shear columns doubled)
void push_forward_voigt(const double W[36], const M3 F, double T[36]) {
    double A[6][6];
    for (int p = 0; p < 6; ++p)
        for (int r = 0; r < 6; ++r) {
            const int i = kVi[p], j = kVj[p], I = kVi[r], Jx = kVj[r];
            A[p][r] = F[i][I] * F[j][Jx] + (r >= 3 ? F[i][Jx] * F[j][I] : 0.0);
        }
    const double J = det3(F);
    double AW[6][6];
    for (int p = 0; p < 6; ++p)
        for (int q = 0; q < 6; ++q) {
            double t = 0.0;
            for (int r = 0; r < 6; ++r) t += A[p][r] * (r <= q ? W[r * 6 + q] : W[q * 6 + r]);  // W upper
            AW[p][q] = t;
        }
    for (int p = 0; p < 6; ++p)
        for (int q = 0; q < 6; ++q) {
            double t = 0.0;
            for (int r = 0; r < 6; ++r) t += AW[p][r] * A[q][r];
            T[p * 6 + q] = t / J;
        }
}

// Neo-Hookean for the Mean Dilatation element (ModNeoHookeanQ1P0.f90): Cauchy stress
// 2 C10 J^(-5/3) (b - tr(b)/3 I) + pbar I with pbar = 3 K (Jbar^(1/3) - 1) / Jbar^(2/3)
// (:429-484); tangent = push-forward of C_iso + C_p (:540-613); params = [C10, BulkModulus].
void nh_q1p0(const double* p, const M3 F, double Jbar, double sig[6], double D[36]) {
    const double C10 = p[0], K = p[1];
    M3 Ft, b, C, Ci;
    transpose3(F, Ft);
    matmul3(F, Ft, b);
    matmul3(Ft, F, C);
    inv3(C, Ci);
    const double trb = b[0][0] + b[1][1] + b[2][2];
    const double J = det3(F);
    const double pbar = (3.0 * K * (std::pow(Jbar, 1.0 / 3.0) - 1.0)) / std::pow(Jbar, 2.0 / 3.0);
    M3 S;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            S[i][j] = 2.0 * C10 * std::pow(J, -5.0 / 3.0) * (b[i][j] - (i == j ? trb / 3.0 : 0.0)) + (i == j ? pbar : 0.0);
    to_voigt(S, sig);
    double CV[6], CinvV[6], SfricV[6] = {2.0 * C10, 2.0 * C10, 2.0 * C10, 0, 0, 0}, devS[6], Siso[6];
    to_voigt(C, CV);
    to_voigt(Ci, CinvV);
    const double sc = inner_voigt(SfricV, CV);
    for (int k = 0; k < 6; ++k) {
        devS[k] = SfricV[k] - (1.0 / 3.0) * sc * CinvV[k];
        Siso[k] = std::pow(J, -2.0 / 3.0) * devS[k];
    }
    double SQ[36], BL[36], B1[36], B2[36], Cbar[36];
    square_voigt(CinvV, CinvV, SQ);
    ball_voigt(CinvV, CinvV, BL);
    ball_voigt(Siso, CinvV, B1);
    ball_voigt(CinvV, Siso, B2);
    for (int k = 0; k < 36; ++k) {
        const double Pm = SQ[k] - (1.0 / 3.0) * BL[k];
        const double Ciso = (2.0 / 3.0) * std::pow(J, -2.0 / 3.0) * sc * Pm - (2.0 / 3.0) * (B1[k] + B2[k]);
        const double Cp = J * pbar * (BL[k] - 2.0 * SQ[k]);
        Cbar[k] = Ciso + Cp;
    }
    push_forward_voigt(Cbar, F, D);
}
// SecondDerivativesOfPSI_Jbar_NeoHookeanQ1P0 (:625-652)
double nh_q1p0_d2psi(const double* p, double Jbar) {
    return -(p[1] * (std::pow(Jbar, 1.0 / 3.0) - 2.0)) / std::pow(Jbar, 5.0 / 3.0);
}

// St Venant-Kirchhoff (ModStVenantKirchhoff.f90:643-780); params = [YoungModulus, Poisson],
// Lambda/Mu from (:238-239).  The reference fills only the upper triangle of D (:751-756);
// the full symmetric D is returned here (the element routine reads the upper triangle).
void svk(const double* p, const M3 F, double sig[6], double D[36]) {
    const double E = p[0], nu = p[1];
    const double Lambda = nu * E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double Mu = E / (2.0 * (1.0 + nu));
    M3 Ft, C, Eg, S, sg;
    transpose3(F, Ft);
    matmul3(Ft, F, C);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Eg[i][j] = 0.5 * (C[i][j] - (i == j ? 1.0 : 0.0));
    const double trE = Eg[0][0] + Eg[1][1] + Eg[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S[i][j] = Lambda * trE * (i == j ? 1.0 : 0.0) + 2.0 * Mu * Eg[i][j];
    pk2_to_cauchy(F, S, sg);
    to_voigt(sg, sig);
    M3 b;
    matmul3(F, Ft, b);
    const double J = det3(F);
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c < 6; ++c) {
            const int i = kVi[a], j = kVj[a], k = kVi[c], l = kVj[c];
            // Cs (:767-772)
            D[a * 6 + c] = (Lambda / J) * b[i][j] * b[k][l] + (Mu / J) * (b[i][k] * b[j][l] + b[i][l] * b[j][k]);
        }
}

// J2 plasticity, small strain (ModJ2Plasticity.f90:385-479 update, :555-620 tangent,
// :625-633 switch).  params = [E, nu, YieldStress, HardeningModulus].
// state = [OldPlasticStrain(6), OldAccumulatedPlasticStrain]; new state same layout.
void j2_small(const double* p, const M3 F, const double* st_old, double* st_new, double sig[6],
              double D[36]) {
    const double E = p[0], nu = p[1], sy = p[2], H = p[3];
    double Strain[6];
    Strain[0] = F[0][0] - 1.0;
    Strain[1] = F[1][1] - 1.0;
    Strain[2] = F[2][2] - 1.0;
    Strain[3] = F[0][1] + F[1][0];
    Strain[4] = F[1][2] + F[2][1];
    Strain[5] = F[0][2] + F[2][0];
    const double K = E / (3.0 * (1.0 - 2.0 * nu));
    const double G = E / (2.0 * (1.0 + nu));
    double Ee_t[6], Edev[6], Sdev_t[6];
    for (int i = 0; i < 6; ++i) Ee_t[i] = Strain[i] - st_old[i];
    const double Evol = Ee_t[0] + Ee_t[1] + Ee_t[2];
    for (int i = 0; i < 6; ++i) Edev[i] = Ee_t[i] - Evol * kDelta[i] / 3.0;
    const double Ep_acum_t = st_old[6];
    const double p_t = K * Evol;
    const double fac[6] = {2, 2, 2, 1, 1, 1};
    for (int i = 0; i < 6; ++i) Sdev_t[i] = G * Edev[i] * fac[i];
    const double q_t = std::sqrt(1.5 * (Sdev_t[0] * Sdev_t[0] + Sdev_t[1] * Sdev_t[1] + Sdev_t[2] * Sdev_t[2] +
                                        2.0 * Sdev_t[3] * Sdev_t[3] + 2.0 * Sdev_t[4] * Sdev_t[4] +
                                        2.0 * Sdev_t[5] * Sdev_t[5]));
    const double phi_t = q_t - (sy + H * Ep_acum_t);
    double dgam = 0.0;
    const bool plastic = !(phi_t <= 0.0);
    if (!plastic) {
        st_new[6] = Ep_acum_t;
        for (int i = 0; i < 6; ++i) st_new[i] = st_old[i];
        for (int i = 0; i < 6; ++i) sig[i] = Sdev_t[i] + p_t * kDelta[i];
    } else {
        dgam = phi_t / (3.0 * G + H);
        double Sdev[6], Ee[6];
        for (int i = 0; i < 6; ++i) Sdev[i] = (1.0 - dgam * 3.0 * G / q_t) * Sdev_t[i];
        for (int i = 0; i < 6; ++i) sig[i] = Sdev[i] + p_t * kDelta[i];
        for (int i = 0; i < 6; ++i) Ee[i] = Sdev[i] / (2.0 * G) + Evol * kDelta[i] / 3.0;
        st_new[6] = st_old[6] + dgam;
        for (int i = 0; i < 6; ++i) st_new[i] = Strain[i] - Ee[i];
    }
    if (!plastic) {
        const double cte = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
        for (int i = 0; i < 36; ++i) D[i] = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) D[i * 6 + j] = cte * (i == j ? 1.0 - nu : nu);
        for (int i = 3; i < 6; ++i) D[i * 6 + i] = cte * (0.5 - nu);
    } else {
        const double nrm = std::sqrt(Sdev_t[0] * Sdev_t[0] + Sdev_t[1] * Sdev_t[1] + Sdev_t[2] * Sdev_t[2] +
                                     2.0 * Sdev_t[3] * Sdev_t[3] + 2.0 * Sdev_t[4] * Sdev_t[4] +
                                     2.0 * Sdev_t[5] * Sdev_t[5]);
        double N[6];
        for (int i = 0; i < 6; ++i) N[i] = Sdev_t[i] / nrm;
        const double c1 = 2.0 * G * (1.0 - dgam * 3.0 * G / q_t);
        const double c2 = 6.0 * G * G * (dgam / q_t - 1.0 / (3.0 * G + H));
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) {
                const double Id = (i == j ? kIsym[i] : 0.0) - kDelta[i] * kDelta[j] / 3.0;
                D[i * 6 + j] = c1 * Id + c2 * N[i] * N[j] + K * kDelta[i] * kDelta[j];
            }
    }
}

// Finite-strain generalized Maxwell (project-defined; no reference implementation).
// Decoupled Neo-Hookean ground state Psi = K/2 (ln J)^2 + mu/2 (I1bar - 3) plus N Maxwell
// branches acting on the isochoric stress, integrated with the recursive update of
// Holzapfel, Nonlinear Solid Mechanics (2000) section 6.10 (after Simo 1987):
//   Q_a^{n+1} = H_a^n + beta_a e^{-xi_a} S_iso^{n+1},
//   H_a^n = e^{-xi_a} (e^{-xi_a} Q_a^n - beta_a S_iso^n),  xi_a = dt / (2 tau_a).
// Material tangent C = C_vol + (1 + sum beta_a e^{-xi_a}) C_iso, pushed forward in closed form.
// params = [mu, K, nb, beta_1, tau_1, ..., beta_4, tau_4];
// state = [S_iso^n (6, Voigt, material), Q_1..Q_nb (6 each)].
void visco_prony(const double* p, const M3 F, double dt, const double* st_old, double* st_new,
                 double sig[6], double D[36]) {
    const double mu = p[0], K = p[1];
    const int nb = (int)p[2];
    M3 Ft, C, Ci, b;
    transpose3(F, Ft);
    matmul3(Ft, F, C);
    matmul3(F, Ft, b);
    inv3(C, Ci);
    const double J = det3(F);
    const double lnJ = std::log(J);
    const double J23 = std::pow(J, -2.0 / 3.0);
    const double trC = C[0][0] + C[1][1] + C[2][2];
    // S_iso = mu J^{-2/3} (I - trC/3 C^{-1})
    M3 Siso;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Siso[i][j] = mu * J23 * ((i == j ? 1.0 : 0.0) - trC / 3.0 * Ci[i][j]);
    double siso_v[6];
    to_voigt(Siso, siso_v);
    double Qsum[6] = {0, 0, 0, 0, 0, 0};
    double delta = 0.0;
    for (int a = 0; a < nb; ++a) {
        const double beta = p[3 + 2 * a], tau = p[4 + 2 * a];
        const double e = std::exp(-dt / (2.0 * tau));
        for (int k = 0; k < 6; ++k) {
            const double Hn = e * (e * st_old[6 + 6 * a + k] - beta * st_old[k]);
            const double Qn1 = Hn + beta * e * siso_v[k];
            st_new[6 + 6 * a + k] = Qn1;
            Qsum[k] += Qn1;
        }
        delta += beta * e;
    }
    for (int k = 0; k < 6; ++k) st_new[k] = siso_v[k];
    // Cauchy: sigma = (K lnJ / J) I + mu/J dev(bbar) + 1/J F Qsum F^T
    M3 Qm, tq, T;
    from_voigt(Qsum, Qm);
    matmul3(Qm, Ft, T);
    matmul3(F, T, tq);
    const double trb = b[0][0] + b[1][1] + b[2][2];
    double tiso[6];
    for (int k = 0; k < 6; ++k) {
        const int i = kVi[k], j = kVj[k];
        tiso[k] = mu * J23 * (b[i][j] - trb / 3.0 * kDelta[k]);
        sig[k] = (K * lnJ / J) * kDelta[k] + tiso[k] / J + tq[i][j] / J;
    }
    // Spatial tangent: c = c_vol + (1+delta) c_iso,
    //  c_vol = K/J I(x)I - 2 K lnJ/J Isym,
    //  J c_iso = 2/3 mu I1bar (Isym - 1/3 I(x)I) - 2/3 (tau_iso(x)I + I(x)tau_iso).
    const double I1b = J23 * trb;
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c < 6; ++c) {
            const double Is = (a == c ? kIsym[a] : 0.0);
            const double vol = (K / J) * kDelta[a] * kDelta[c] - 2.0 * (K * lnJ / J) * Is;
            const double iso = (2.0 / 3.0) * mu * I1b * (Is - kDelta[a] * kDelta[c] / 3.0) -
                               (2.0 / 3.0) * (tiso[a] * kDelta[c] + kDelta[a] * tiso[c]);
            D[a * 6 + c] = vol + (1.0 + delta) * iso / J;
        }
}

// Multiplicative finite-strain J2 plasticity with a Neo-Hookean elastic response in b_e
// and linear isotropic hardening (project-defined; no reference implementation).
// Algorithm: Simo (1988) / Simo & Hughes, Computational Inelasticity (1998), Box 9.1:
// trial b_e = F Cp^{-1} F^T, radial return on s = mu dev(bbar_e), U(J) = K/2 (1/2 (J^2-1) - ln J).
// The return mapping (closed form for linear hardening) runs in FP64.  The consistent
// spatial tangent is the algorithmic one of Simo (1988) (Simo & Hughes 1998, Box 9.2), formed on
// the Kirchhoff stress and divided by J: volumetric K J^2 1(x)1 - K (J^2 - 1) I, the trial
// deviatoric modulus 2 mubar (I - 1(x)1/3) - 2/3 (s(x)1 + 1(x)s), and, when plastic, that
// modulus scaled by (1 - beta1) with the rank-one return-mapping corrections in n.  It is not
// symmetric and is symmetrized (D + D^T)/2 because the global matrix is stored symmetric.
// params = [E, nu, sigma_y0, H]; state = [Cp^{-1} (Voigt 6), alpha].
void j2_finite(const double* p, const M3 F, const double* st_old, double* st_new, double sig[6],
               double D[36], double* Dfull /* may be NULL: unsymmetrized tangent */) {
    const double E = p[0], nu = p[1], sy = p[2], H = p[3];
    const double mu = E / (2.0 * (1.0 + nu));
    const double K = E / (3.0 * (1.0 - 2.0 * nu));
    M3 Cpi, Ft, T, be;
    from_voigt(st_old, Cpi);
    transpose3(F, Ft);
    matmul3(Cpi, Ft, T);
    matmul3(F, T, be);
    const double J = det3(F);
    const double J23 = std::pow(J, -2.0 / 3.0);
    const double trbe = J23 * (be[0][0] + be[1][1] + be[2][2]);
    const double Ie = trbe / 3.0;
    const double mub = mu * Ie;
    double s[6];
    for (int k = 0; k < 6; ++k) s[k] = mu * (J23 * be[kVi[k]][kVj[k]] - Ie * kDelta[k]);
    const double ns = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2] +
                                2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
    const double alpha = st_old[6];
    const double f = ns - std::sqrt(2.0 / 3.0) * (sy + H * alpha);
    const bool plastic = f > 0.0;
    double n[6] = {0, 0, 0, 0, 0, 0};
    double beta1 = 0.0, g = 0.0;
    if (ns > 0.0)
        for (int k = 0; k < 6; ++k) n[k] = s[k] / ns;
    double snew[6];
    if (plastic) {
        g = 3.0 * mub * f / (3.0 * mub + H);  // 2 mubar dgamma
        beta1 = g / ns;
        for (int k = 0; k < 6; ++k) snew[k] = s[k] - g * n[k];
        st_new[6] = alpha + std::sqrt(2.0 / 3.0) * g / (2.0 * mub);
    } else {
        for (int k = 0; k < 6; ++k) snew[k] = s[k];
        st_new[6] = alpha;
    }
    // bbar_e^{n+1} = s/mu + Ie I; Cp^{-1} = F^{-1} J^{2/3} bbar_e F^{-T}
    M3 bbn, Fi, Fit, T2, Cpn;
    double bbv[6];
    for (int k = 0; k < 6; ++k) bbv[k] = snew[k] / mu + Ie * kDelta[k];
    from_voigt(bbv, bbn);
    inv3(F, Fi);
    transpose3(Fi, Fit);
    matmul3(bbn, Fit, T2);
    matmul3(Fi, T2, Cpn);
    const double Jm23 = 1.0 / J23;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Cpn[i][j] *= Jm23;
    double cpv[6];
    to_voigt(Cpn, cpv);
    for (int k = 0; k < 6; ++k) st_new[k] = cpv[k];
    // Cauchy stress
    const double Jp = 0.5 * K * (J * J - 1.0);
    for (int k = 0; k < 6; ++k) sig[k] = (Jp * kDelta[k] + snew[k]) / J;
    // Tangent (Kirchhoff-based, divided by J at the end)
    double n2[6];
    {
        M3 nm, nn;
        from_voigt(n, nm);
        matmul3(nm, nm, nn);
        to_voigt(nn, n2);
    }
    double A[36];
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c < 6; ++c) {
            const double Is = (a == c ? kIsym[a] : 0.0);
            const double dev = 2.0 * mub * (Is - kDelta[a] * kDelta[c] / 3.0) -
                               (2.0 / 3.0) * (s[a] * kDelta[c] + kDelta[a] * s[c]);
            double v = dev;
            if (plastic) {
                const double b0inv = 3.0 * mub / (3.0 * mub + H);
                const double cH = 2.0 * f * H * ns / ((3.0 * mub + H) * (3.0 * mub + H));
                const double vc = 2.0 * mub * n[c] - (2.0 / 3.0) * ns * kDelta[c] + 2.0 * ns * n2[c];
                v = (1.0 - beta1) * dev - n[a] * ((b0inv - beta1) * vc + cH * n[c]);
            }
            A[a * 6 + c] = K * J * J * kDelta[a] * kDelta[c] - K * (J * J - 1.0) * Is + v;
        }
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c < 6; ++c) {
            D[a * 6 + c] = 0.5 * (A[a * 6 + c] + A[c * 6 + a]) / J;
            if (Dfull) Dfull[a * 6 + c] = A[a * 6 + c] / J;
        }
}

}  // namespace

// =========================================================================================
// Public material-point API
// =========================================================================================
extern "C" int or_model_nparams(int model) {
    switch (model) {
        case OR_CNH: return 2;
        case OR_NH_Q1P0: return 2;
        case OR_SVK: return 2;
        case OR_J2_SMALL: return 4;
        case OR_VISCO_VAR: return 6;
        case OR_VISCO_PRONY: return 11;
        case OR_J2_FINITE: return 4;
    }
    return -1;
}

extern "C" int or_model_nstate(int model) {
    switch (model) {
        case OR_CNH: return 0;
        case OR_NH_Q1P0: return 0;
        case OR_SVK: return 0;
        case OR_J2_SMALL: return 7;
        case OR_VISCO_VAR: return 19;
        case OR_VISCO_PRONY: return 6 + 6 * 4;
        case OR_J2_FINITE: return 7;
    }
    return -1;
}

extern "C" void or_model_init_state(int model, const double* params, double* st) {
    const int ns = or_model_nstate(model);
    for (int i = 0; i < ns; ++i) st[i] = 0.0;
    (void)params;
    if (model == OR_J2_FINITE) { st[0] = st[1] = st[2] = 1.0; }
    if (model == OR_VISCO_VAR) {  // Fv_old = I (ModViscoelasticMatrix.f90:124-131)
        st[0] = st[4] = st[8] = 1.0;
    }
}

int visco_var_update(const double* p, const double* F, double dt, const double* st_old,
                     double* st_new, double* sig, double* D);  // ceos_oracle_visco.cpp

extern "C" int or_material_point(int model, const double* params, const double* Fin, double dt,
                                 const double* st_old, double* st_new, double* sigma, double* D) {
    M3 F;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = Fin[i * 3 + j];
    switch (model) {
        case OR_CNH: cnh(params, F, sigma, D); return 0;
        case OR_NH_Q1P0: nh_q1p0(params, F, det3(F), sigma, D); return 0;  // single point: Jbar = J
        case OR_SVK: svk(params, F, sigma, D); return 0;
        case OR_J2_SMALL: j2_small(params, F, st_old, st_new, sigma, D); return 0;
        case OR_VISCO_PRONY: visco_prony(params, F, dt, st_old, st_new, sigma, D); return 0;
        case OR_J2_FINITE: j2_finite(params, F, st_old, st_new, sigma, D, nullptr); return 0;
        case OR_VISCO_VAR: return visco_var_update(params, Fin, dt, st_old, st_new, sigma, D);
    }
    return 9;
}

// Unsymmetrized J2-finite tangent, for the finite-difference consistency test.
extern "C" int or_j2_finite_full_tangent(const double* params, const double* Fin, const double* st_old,
                                         double* st_new, double* sigma, double* Dfull) {
    M3 F;
    double D[36];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = Fin[i * 3 + j];
    j2_finite(params, F, st_old, st_new, sigma, D, Dfull);
    return 0;
}

// =========================================================================================
// CSR pattern (ModFEMAnalysis.f90:209-273; ModSparseMatrixRoutines.f90:254-288, 573-609;
// ModSparseVectorRoutines.f90:222-312).  Every element sets the block GM x GM of ones;
// AddItems keeps each row as a sorted list of distinct columns.  The upper-triangle
// conversion keeps col >= row, nz = (nz_full - n)/2 + n, RowMap(n+1) = nz+1 (1-based).
// =========================================================================================
namespace {
void element_gm(const int* conn, int e, int GM[24]) {  // GetGlobalMapping (ModElement.f90:1550-1591)
    for (int n = 0; n < 8; ++n)
        for (int d = 0; d < 3; ++d) GM[3 * n + d] = 3 * (conn[8 * e + n] - 1) + d + 1;
}

void build_rows(int n_nodes, int n_elem, const int* conn, std::vector<std::vector<int>>& rows) {
    const int n = 3 * n_nodes;
    rows.assign(n, {});
    int GM[24];
    for (int e = 0; e < n_elem; ++e) {
        element_gm(conn, e, GM);
        int ordem[24];
        std::copy(GM, GM + 24, ordem);
        std::sort(ordem, ordem + 24);  // organizar(cols)
        for (int i = 0; i < 24; ++i) {
            std::vector<int>& r = rows[GM[i] - 1];
            for (int k = 0; k < 24; ++k) {  // AddItems: sorted insert of distinct columns
                auto it = std::lower_bound(r.begin(), r.end(), ordem[k]);
                if (it == r.end() || *it != ordem[k]) r.insert(it, ordem[k]);
            }
        }
    }
}
}  // namespace

extern "C" long long or_pattern_nnz(int n_nodes, int n_elem, const int* conn) {
    std::vector<std::vector<int>> rows;
    build_rows(n_nodes, n_elem, conn, rows);
    long long nz = 0;
    for (auto& r : rows) nz += (long long)r.size();
    const long long n = 3LL * n_nodes;
    return (nz - n) / 2 + n;
}

extern "C" void or_pattern_fill(int n_nodes, int n_elem, const int* conn, int* rowmap, int* col, int* row) {
    std::vector<std::vector<int>> rows;
    build_rows(n_nodes, n_elem, conn, rows);
    const int n = 3 * n_nodes;
    long long nz = 0;
    for (auto& r : rows) nz += (long long)r.size();
    nz = (nz - n) / 2 + n;
    long long k = 0;
    for (int irow = 1; irow <= n; ++irow) {
        rowmap[irow - 1] = (int)(k + 1);
        for (int c : rows[irow - 1])
            if (c >= irow) {
                if (col) col[k] = c;
                if (row) row[k] = irow;
                ++k;
            }
    }
    rowmap[n] = (int)(nz + 1);
}

extern "C" void or_slot_map(int n_nodes, int n_elem, const int* conn, const int* rowmap, const int* col,
                            long long* out) {
    (void)n_nodes;
    int GM[24];
    for (int e = 0; e < n_elem; ++e) {
        element_gm(conn, e, GM);
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) {
                long long pos = -1;
                const int iG = GM[i], jG = GM[j];
                if (jG >= iG) {
                    // linear search of SubAssembleGlobalMatrixUpperTriangular.f90:51-56
                    for (int k = rowmap[iG - 1]; k <= rowmap[iG] - 1; ++k)
                        if (col[k - 1] == jG) pos = k - 1;
                    if (pos < 0) std::abort();  // "Assembly error :: KgRowMap position not found"
                }
                out[((long long)e * 24 + i) * 24 + j] = pos;
            }
    }
}

// =========================================================================================
// Model object and the element loop
// =========================================================================================
struct or_model {
    int n_nodes, n_elem, n_mat, per_element, n_params_max, nstate;
    std::vector<double> X;
    std::vector<int> conn, mat_id, models;
    std::vector<double> params;
    std::vector<int> rowmap, col;
    long long nnz;
    // Gauss-point storage (8 per element)
    std::vector<double> st_old, st_new;   // [n_elem*8*nstate]
    std::vector<double> sigma;            // [n_elem*8*6]
    std::vector<double> Dgp;              // [n_elem*8*36]
    std::vector<int> gp_status;
    std::vector<double> jbar, vol0;       // [n_elem] Mean Dilatation: V/V0 and V0 of the last update
    double time_old = 0.0;
    const double* elem_params(int e) const {
        return per_element ? &params[(size_t)e * n_params_max] : &params[(size_t)mat_id[e] * n_params_max];
    }
    int elem_model(int e) const { return models[mat_id[e]]; }
};

extern "C" or_model* or_create(int n_nodes, int n_elem, const double* X, const int* conn, const int* mat_id,
                               int n_mat, const int* models, int per_element, int n_params_max,
                               const double* params) {
    or_model* m = new or_model();
    m->n_nodes = n_nodes;
    m->n_elem = n_elem;
    m->n_mat = n_mat;
    m->per_element = per_element;
    m->n_params_max = n_params_max;
    m->X.assign(X, X + 3 * (size_t)n_nodes);
    m->conn.assign(conn, conn + 8 * (size_t)n_elem);
    m->mat_id.assign(mat_id, mat_id + n_elem);
    m->models.assign(models, models + n_mat);
    m->params.assign(params, params + (size_t)(per_element ? n_elem : n_mat) * n_params_max);
    int ns = 0;
    for (int k = 0; k < n_mat; ++k) ns = std::max(ns, or_model_nstate(models[k]));
    m->nstate = ns;
    m->nnz = or_pattern_nnz(n_nodes, n_elem, conn);
    m->rowmap.resize(3 * (size_t)n_nodes + 1);
    m->col.resize(m->nnz);
    or_pattern_fill(n_nodes, n_elem, conn, m->rowmap.data(), m->col.data(), nullptr);
    const size_t ngp = (size_t)n_elem * 8;
    m->st_old.assign(ngp * ns, 0.0);
    m->st_new.assign(ngp * ns, 0.0);
    for (int e = 0; e < n_elem; ++e)
        for (int g = 0; g < 8; ++g) {
            or_model_init_state(m->elem_model(e), m->elem_params(e), &m->st_old[((size_t)e * 8 + g) * ns]);
            or_model_init_state(m->elem_model(e), m->elem_params(e), &m->st_new[((size_t)e * 8 + g) * ns]);
        }
    m->sigma.assign(ngp * 6, 0.0);
    m->Dgp.assign(ngp * 36, 0.0);
    m->gp_status.assign(ngp, 0);
    m->jbar.assign(n_elem, 1.0);
    m->vol0.assign(n_elem, 1.0);
    return m;
}

extern "C" void or_destroy(or_model* m) { delete m; }
extern "C" long long or_nnz(or_model* m) { return m->nnz; }
extern "C" void or_get_pattern(or_model* m, int* rowmap, int* col) {
    std::copy(m->rowmap.begin(), m->rowmap.end(), rowmap);
    std::copy(m->col.begin(), m->col.end(), col);
}

namespace {

// Jacobian of the reference or current coordinates: Jacob(i,j) = sum_n dN(n,i) * x_n(j)
void jacobian(const double dN[8][3], const double xe[8][3], M3 Jac) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int n = 0; n < 8; ++n) s += dN[n][i] * xe[n][j];
            Jac[i][j] = s;
        }
}
// DifSf(n,:) = matmul(inverse(Jacob), DifSf(n,:))
void global_derivs(const M3 Jinv, const double dN[8][3], double dNx[8][3]) {
    for (int n = 0; n < 8; ++n)
        for (int j = 0; j < 3; ++j) dNx[n][j] = Jinv[j][0] * dN[n][0] + Jinv[j][1] * dN[n][1] + Jinv[j][2] * dN[n][2];
}

struct ElemGeom {
    double Xe[8][3], xe[8][3], ue[24];
};

void gather(const or_model* m, int e, const double* U, ElemGeom& g) {
    for (int n = 0; n < 8; ++n) {
        const int node = m->conn[8 * e + n] - 1;
        for (int d = 0; d < 3; ++d) {
            g.Xe[n][d] = m->X[3 * node + d];
            g.ue[3 * n + d] = U[3 * node + d];
            g.xe[n][d] = g.Xe[n][d] + g.ue[3 * n + d];  // UpdateMeshCoordinates: Coord = CoordX + U
        }
    }
}

// SolveConstitutiveModel for one element (FEM/Subroutines/SubSolveConstitutiveModel.f90:56-136):
// ElementVolume (ModElement.f90:1313-1427), DeformationGradient (:1210-1300), model update.
int element_update(or_model* m, int e, const ElemGeom& g, double dt) {
    int status = 0;
    // ElementVolume: detJ (current) <= 1e-13 is an error
    for (int gp = 0; gp < 8; ++gp) {
        double xi[3], w, dN[8][3];
        hexa8_gp(gp, xi, &w);
        hexa8_dN(xi, dN);
        M3 Jc;
        jacobian(dN, g.xe, Jc);
        if (det3(Jc) <= 1.0e-13) status = 1;
    }
    const int ns = m->nstate;
    const bool q1p0 = m->elem_model(e) == OR_NH_Q1P0;
    if (q1p0) {  // Jbar = Volume / VolumeX for every Gauss point (SubSolveConstitutiveModel.f90:65,100)
        double V = 0.0, V0 = 0.0;
        for (int gp = 0; gp < 8; ++gp) {
            double xi[3], w, dN[8][3];
            hexa8_gp(gp, xi, &w);
            hexa8_dN(xi, dN);
            M3 Jc, JX;
            jacobian(dN, g.xe, Jc);
            jacobian(dN, g.Xe, JX);
            V0 += w * det3(JX);
            V += w * det3(Jc);
        }
        m->jbar[e] = V / V0;
        m->vol0[e] = V0;
    }
    for (int gp = 0; gp < 8; ++gp) {
        double xi[3], w, dN[8][3], dNX[8][3];
        hexa8_gp(gp, xi, &w);
        hexa8_dN(xi, dN);
        M3 JX, JXi;
        jacobian(dN, g.Xe, JX);
        if (det3(JX) <= 1.0e-13) { status = 1; continue; }
        inv3(JX, JXi);
        global_derivs(JXi, dN, dNX);
        double F[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int n = 0; n < 8; ++n) s += dNX[n][j] * g.ue[3 * n + i];
                F[i * 3 + j] = s + (i == j ? 1.0 : 0.0);
            }
        const size_t q = (size_t)e * 8 + gp;
        int st = 0;
        if (q1p0) {
            M3 Fm;
            for (int i = 0; i < 9; ++i) Fm[i / 3][i % 3] = F[i];
            nh_q1p0(m->elem_params(e), Fm, m->jbar[e], &m->sigma[q * 6], &m->Dgp[q * 36]);
        } else {
            st = or_material_point(m->elem_model(e), m->elem_params(e), F, dt, &m->st_old[q * ns],
                                   &m->st_new[q * ns], &m->sigma[q * 6], &m->Dgp[q * 36]);
        }
        m->gp_status[q] = st;
        if (st && !status) status = st;
    }
    return status;
}

// Matrix_B_and_G / MatrixBG_ThreeDimensional (ModElement.f90:787-889) on current coordinates.
bool bg_matrices(const ElemGeom& g, int gp, double B[6][24], double G[9][24], double* detJ, double* w) {
    double xi[3], dN[8][3], dNx[8][3];
    hexa8_gp(gp, xi, w);
    hexa8_dN(xi, dN);
    M3 Jc, Jci;
    jacobian(dN, g.xe, Jc);
    *detJ = det3(Jc);
    if (*detJ <= 1.0e-13) return false;
    inv3(Jc, Jci);
    global_derivs(Jci, dN, dNx);
    std::memset(B, 0, sizeof(double) * 6 * 24);
    std::memset(G, 0, sizeof(double) * 9 * 24);
    for (int n = 0; n < 8; ++n) {
        const int c = 3 * n;
        B[0][c] = dNx[n][0];
        B[1][c + 1] = dNx[n][1];
        B[2][c + 2] = dNx[n][2];
        B[3][c] = dNx[n][1]; B[3][c + 1] = dNx[n][0];
        B[4][c + 2] = dNx[n][1]; B[4][c + 1] = dNx[n][2];
        B[5][c + 2] = dNx[n][0]; B[5][c] = dNx[n][2];
        for (int d = 0; d < 3; ++d)
            for (int k = 0; k < 3; ++k) G[3 * d + k][c + d] = dNx[n][k];
    }
    return true;
}

// ElementInternalForce (ModElement.f90:484-563): Fe += w detJ B^T sigma
int element_fint(const or_model* m, int e, const ElemGeom& g, double Fe[24]) {
    for (int i = 0; i < 24; ++i) Fe[i] = 0.0;
    for (int gp = 0; gp < 8; ++gp) {
        double B[6][24], G[9][24], detJ, w;
        if (!bg_matrices(g, gp, B, G, &detJ, &w)) return 1;
        const double* s = &m->sigma[((size_t)e * 8 + gp) * 6];
        const double a = w * detJ;
        for (int c = 0; c < 24; ++c) {
            double t = 0.0;
            for (int r = 0; r < 6; ++r) t += B[r][c] * s[r];
            Fe[c] += a * t;
        }
    }
    return 0;
}

// ElementStiffnessMatrix, nonlinear full integration (ModElement.f90:310-348):
// Ke += w detJ (B^T (D B) + G^T (S G)); D and S are read through their upper triangle
// (dsymm 'L','U', ModMathRoutines.f90:975-1000); S = blockdiag(sigma) (ModConstitutiveModel.f90:292-314).
// Mean Dilatation (ModElement.f90:429-469) adds Bdiv^T Bdiv d2psi/dJbar2 / VolumeX with
// Bdiv = sum_gp w detJ (G(1,:) + G(5,:) + G(9,:)).
void element_stiffness(const or_model* m, int e, const ElemGeom& g, double Ke[24][24]) {
    std::memset(Ke, 0, sizeof(double) * 576);
    const bool q1p0 = m->elem_model(e) == OR_NH_Q1P0;
    double Bdiv[24] = {0};
    for (int gp = 0; gp < 8; ++gp) {
        double B[6][24], G[9][24], detJ, w;
        if (!bg_matrices(g, gp, B, G, &detJ, &w)) continue;
        if (q1p0)
            for (int c = 0; c < 24; ++c) Bdiv[c] += (G[0][c] + G[4][c] + G[8][c]) * w * detJ;
        const double* Dg = &m->Dgp[((size_t)e * 8 + gp) * 36];
        const double* s = &m->sigma[((size_t)e * 8 + gp) * 6];
        double Ds[6][6], S[9][9];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) Ds[i][j] = (i <= j) ? Dg[i * 6 + j] : Dg[j * 6 + i];
        double sm[3][3];
        from_voigt(s, sm);
        std::memset(S, 0, sizeof(S));
        for (int b = 0; b < 3; ++b)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) S[3 * b + i][3 * b + j] = sm[i][j];
        double DB[6][24], SG[9][24];
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 24; ++c) {
                double t = 0.0;
                for (int k = 0; k < 6; ++k) t += Ds[i][k] * B[k][c];
                DB[i][c] = t;
            }
        for (int i = 0; i < 9; ++i)
            for (int c = 0; c < 24; ++c) {
                double t = 0.0;
                for (int k = 0; k < 9; ++k) t += S[i][k] * G[k][c];
                SG[i][c] = t;
            }
        const double a = w * detJ;
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) {
                double t = 0.0;
                for (int k = 0; k < 6; ++k) t += B[k][i] * DB[k][j];
                Ke[i][j] += a * t;
            }
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) {
                double t = 0.0;
                for (int k = 0; k < 9; ++k) t += G[k][i] * SG[k][j];
                Ke[i][j] += a * t;
            }
    }
    if (q1p0) {
        const double kd = nh_q1p0_d2psi(m->elem_params(e), m->jbar[e]) / m->vol0[e];
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) Ke[i][j] += Bdiv[i] * Bdiv[j] * kd;
    }
}

// AssembleGlobalMatrixUpperTriangular (SubAssembleGlobalMatrixUpperTriangular.f90:43-65)
void assemble_upper(const or_model* m, const int GM[24], const double Ke[24][24], double* kval) {
    for (int i = 0; i < 24; ++i) {
        const int iG = GM[i];
        for (int j = 0; j < 24; ++j) {
            const int jG = GM[j];
            if (jG >= iG) {
                bool found = false;
                for (int k = m->rowmap[iG - 1]; k <= m->rowmap[iG] - 1; ++k)
                    if (m->col[k - 1] == jG) {
                        found = true;
                        kval[k - 1] += Ke[i][j];
                    }
                if (!found) std::abort();
            }
        }
    }
}

}  // namespace

extern "C" int or_evaluate(or_model* m, double time, const double* U, double* fint, double* kval,
                           int* n_failed, int* failed_ids) {
    const double dt = time - m->time_old;
    int status = 0, nf = 0;
    ElemGeom g;
    // SolveConstitutiveModel
    std::vector<char> failed(m->n_elem, 0);
    for (int e = 0; e < m->n_elem; ++e) {
        gather(m, e, U, g);
        const int st = element_update(m, e, g, dt);
        if (st) {
            failed[e] = 1;
            if (!status) status = st;
        }
    }
    // InternalForce (SubInternalForce.f90:53-85)
    const int n = 3 * m->n_nodes;
    for (int i = 0; i < n; ++i) fint[i] = 0.0;
    for (int e = 0; e < m->n_elem; ++e) {
        gather(m, e, U, g);
        double Fe[24];
        int GM[24];
        element_gm(m->conn.data(), e, GM);
        if (element_fint(m, e, g, Fe)) {
            failed[e] = 1;
            if (!status) status = 1;
        }
        for (int i = 0; i < 24; ++i) fint[GM[i] - 1] += Fe[i];
    }
    // TangentStiffnessMatrix, FEM branch (SubTangentStiffnessMatrix.f90:63, 294-311)
    if (kval) {
        for (long long k = 0; k < m->nnz; ++k) kval[k] = 0.0;
        for (int e = 0; e < m->n_elem; ++e) {
            gather(m, e, U, g);
            double Ke[24][24];
            int GM[24];
            element_gm(m->conn.data(), e, GM);
            element_stiffness(m, e, g, Ke);
            assemble_upper(m, GM, Ke, kval);
        }
    }
    for (int e = 0; e < m->n_elem; ++e)
        if (failed[e]) {
            if (failed_ids) failed_ids[nf] = e + 1;
            ++nf;
        }
    if (n_failed) *n_failed = nf;
    return status;
}

// CPU baseline: the same three passes on the first n_eval elements, optionally on OpenMP
// threads with elements coloured into 8 classes (parity of the element's structured
// (i,j,k) position is not known for general meshes, so colours are built greedily by node
// conflicts) so that the scatter needs no atomics.
extern "C" int or_evaluate_sample(or_model* m, double time, const double* U, double* fint, double* kval,
                                  int n_eval, int threads) {
    const double dt = time - m->time_old;
    n_eval = std::min(n_eval, m->n_elem);
    const int n = 3 * m->n_nodes;
    for (int i = 0; i < n; ++i) fint[i] = 0.0;
    if (kval)
        for (long long k = 0; k < m->nnz; ++k) kval[k] = 0.0;
    // greedy colouring
    static thread_local std::vector<int> colour_of;
    static thread_local std::vector<std::vector<int>> classes;
    static thread_local int coloured_for = -1;
    if (coloured_for != n_eval || (int)colour_of.size() != n_eval) {
        colour_of.assign(n_eval, -1);
        classes.clear();
        std::vector<std::vector<int>> node_colours(m->n_nodes);
        for (int e = 0; e < n_eval; ++e) {
            unsigned long long used = 0;
            for (int a = 0; a < 8; ++a)
                for (int c : node_colours[m->conn[8 * e + a] - 1]) used |= 1ULL << c;
            int c = 0;
            while (used & (1ULL << c)) ++c;
            colour_of[e] = c;
            if ((int)classes.size() <= c) classes.resize(c + 1);
            classes[c].push_back(e);
            for (int a = 0; a < 8; ++a) node_colours[m->conn[8 * e + a] - 1].push_back(c);
        }
        coloured_for = n_eval;
    }
    int status = 0;
#ifdef _OPENMP
    if (threads < 1) threads = 1;
#endif
    for (auto& cls : classes) {
        const int nc = (int)cls.size();
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static) reduction(max : status)
#endif
        for (int t = 0; t < nc; ++t) {
            const int e = cls[t];
            ElemGeom g;
            gather(m, e, U, g);
            int st = element_update(m, e, g, dt);
            double Fe[24];
            int GM[24];
            element_gm(m->conn.data(), e, GM);
            if (element_fint(m, e, g, Fe)) st = 1;
            for (int i = 0; i < 24; ++i) fint[GM[i] - 1] += Fe[i];
            if (kval) {
                double Ke[24][24];
                element_stiffness(m, e, g, Ke);
                assemble_upper(m, GM, Ke, kval);
            }
            if (st > status) status = st;
        }
    }
    (void)threads;
    return status;
}

// HomogenizeStress (MultiScale/ModMultiscaleAnalysis.f90:140-329): Pbar = (1/V0) sum_e sum_gp
// P w detJ_X with P = J sigma F^{-T} (StressTransformation Cauchy -> FirstPiola) of the Gauss-point
// stresses of the last evaluation, F recomputed from U, V0 = sum of the element reference volumes.
// P_out: row-major 3x3.
extern "C" void or_homogenize(or_model* m, const double* U, double* P_out) {
    double P[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double V0 = 0.0;
    ElemGeom g;
    for (int e = 0; e < m->n_elem; ++e) {
        gather(m, e, U, g);
        for (int gp = 0; gp < 8; ++gp) {
            double xi[3], w, dN[8][3], dNX[8][3];
            hexa8_gp(gp, xi, &w);
            hexa8_dN(xi, dN);
            M3 JX, JXi;
            jacobian(dN, g.Xe, JX);
            const double detJX = det3(JX);
            V0 += w * detJX;
            inv3(JX, JXi);
            global_derivs(JXi, dN, dNX);
            M3 F, Fi, sg;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int n = 0; n < 8; ++n) s += dNX[n][j] * g.ue[3 * n + i];
                    F[i][j] = s + (i == j ? 1.0 : 0.0);
                }
            inv3(F, Fi);
            from_voigt(&m->sigma[((size_t)e * 8 + gp) * 6], sg);
            const double J = det3(F);
            for (int i = 0; i < 3; ++i)
                for (int Jc = 0; Jc < 3; ++Jc) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += sg[i][k] * Fi[Jc][k];  // sigma F^{-T}
                    P[i][Jc] += w * detJX * J * s;
                }
        }
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P_out[3 * i + j] = P[i][j] / V0;
}

extern "C" void or_commit(or_model* m) {
    m->st_old = m->st_new;  // SwitchConvergedState (ModFEMAnalysis.f90:1349-1353)
}
extern "C" void or_set_time_old(or_model* m, double t) { m->time_old = t; }
extern "C" void or_get_gp_stress(or_model* m, double* sigma) { std::copy(m->sigma.begin(), m->sigma.end(), sigma); }
extern "C" int or_get_state(or_model* m, double* st, int which) {
    const auto& v = which ? m->st_new : m->st_old;
    std::copy(v.begin(), v.end(), st);
    return m->nstate;
}
extern "C" int or_set_state(or_model* m, const double* st, int which) {
    auto& v = which ? m->st_new : m->st_old;
    std::copy(st, st + v.size(), v.begin());
    return m->nstate;
}

// =========================================================================================
// Host driver: boundary conditions, Newton-Raphson, quasi-static increments
// =========================================================================================
namespace {

// Skyline (variable-band) LDL^T factorization of the symmetric matrix given by its upper
// CSR, used in place of PARDISO (which is unavailable).  Columns stored from their first
// nonzero row to the diagonal.
struct Skyline {
    int n;
    std::vector<long long> colptr;  // start of column j in a[]
    std::vector<int> top;           // first row of column j
    std::vector<double> a;
    void build(int n_, const int* rowmap, const int* col, const double* val) {
        n = n_;
        top.assign(n, 0);
        for (int j = 0; j < n; ++j) top[j] = j;
        for (int r = 0; r < n; ++r)
            for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
                const int c = col[k] - 1;
                if (r < top[c]) top[c] = r;
            }
        colptr.assign(n + 1, 0);
        for (int j = 0; j < n; ++j) colptr[j + 1] = colptr[j] + (j - top[j] + 1);
        a.assign(colptr[n], 0.0);
        for (int r = 0; r < n; ++r)
            for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
                const int c = col[k] - 1;
                at(r, c) += val[k];
            }
    }
    double& at(int i, int j) { return a[colptr[j] + (i - top[j])]; }  // i <= j, i >= top[j]
    bool factor() {
        for (int j = 0; j < n; ++j) {
            // g_ij = a_ij - sum_{k<i} l_ki g_kj, for i in [top_j, j)
            for (int i = top[j]; i < j; ++i) {
                const int k0 = std::max(top[i], top[j]);
                double s = 0.0;
                for (int k = k0; k < i; ++k) s += at(k, i) * at(k, j);
                at(i, j) -= s;
            }
            double d = at(j, j);
            for (int i = top[j]; i < j; ++i) {
                const double g = at(i, j);
                const double l = g / at(i, i);
                d -= l * g;
                at(i, j) = l;
            }
            if (d == 0.0 || !std::isfinite(d)) return false;
            at(j, j) = d;
        }
        return true;
    }
    void solve(double* x) {
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int i = top[j]; i < j; ++i) s += at(i, j) * x[i];
            x[j] -= s;
        }
        for (int j = 0; j < n; ++j) x[j] /= at(j, j);
        for (int j = n - 1; j >= 0; --j)
            for (int i = top[j]; i < j; ++i) x[i] -= at(i, j) * x[j];
    }
};

// y = K x with K symmetric given by its upper triangle (mkl_dcsrsymv 'U').
void symv_upper(int n, const int* rowmap, const int* col, const double* val, const double* x, double* y) {
    for (int i = 0; i < n; ++i) y[i] = 0.0;
    for (int r = 0; r < n; ++r)
        for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
            const int c = col[k] - 1;
            y[r] += val[k] * x[c];
            if (c != r) y[c] += val[k] * x[r];
        }
}

}  // namespace

extern "C" int or_analysis(or_model* m, int n_steps, const double* step_t0, const double* step_dt, int n_fixed,
                           const int* fixed_dofs, int n_presc, const int* presc_dofs, const double* presc_init,
                           const double* presc_final, int n_force, const int* force_dofs, const double* force_init,
                           const double* force_final, double tol, int itmax, int norm_mode, int norm_type,
                           int max_cutbacks, int* iters, int* cutbacks, int n_probe, const int* probe_dofs,
                           double* probe_out, int max_log, double* norm_log, int* n_log, double* U_final) {
    const int n = 3 * m->n_nodes;
    const long long nnz = m->nnz;
    std::vector<double> U(n, 0.0), Uconv(n), Ubar(n), Ubar0(n), Fext(n), Fext0(n), dFext(n), dUp(n);
    std::vector<double> X(n), R(n), fint(n), kval(nnz), DX(n), Ud(n), Rmod(n);
    // zero / one masks (AllocatePrescDispSparseMapping, ModBoundaryConditions.f90:344-440 and the
    // fixed-support twin): entries whose row or column is constrained, and their diagonals.
    std::vector<char> is_presc(n, 0), is_fixed(n, 0);
    for (int i = 0; i < n_presc; ++i) is_presc[presc_dofs[i] - 1] = 1;
    for (int i = 0; i < n_fixed; ++i) is_fixed[fixed_dofs[i] - 1] = 1;
    std::vector<long long> zp, op, zf, of;
    for (int r = 0; r < n; ++r)
        for (int k = m->rowmap[r] - 1; k < m->rowmap[r + 1] - 1; ++k) {
            const int c = m->col[k] - 1;
            if (is_presc[r] || is_presc[c]) zp.push_back(k);
            if (is_presc[r] && c == r) op.push_back(k);
            if (is_fixed[r] || is_fixed[c]) zf.push_back(k);
            if (is_fixed[r] && c == r) of.push_back(k);
        }
    const double GR = (1.0 + std::sqrt(5.0)) / 2.0;
    int nl = 0;
    for (int ST = 0; ST < n_steps; ++ST) {
        // GetBoundaryConditions: Fext = initial, DeltaFext = final - initial, U(presc) = initial
        std::fill(Fext0.begin(), Fext0.end(), 0.0);
        std::fill(dFext.begin(), dFext.end(), 0.0);
        for (int i = 0; i < n_force; ++i) {
            Fext0[force_dofs[i] - 1] += force_init[(size_t)i * n_steps + ST];
            dFext[force_dofs[i] - 1] += force_final[(size_t)i * n_steps + ST] - force_init[(size_t)i * n_steps + ST];
        }
        std::fill(dUp.begin(), dUp.end(), 0.0);
        for (int i = 0; i < n_presc; ++i) {
            U[presc_dofs[i] - 1] = presc_init[(size_t)i * n_steps + ST];
            dUp[presc_dofs[i] - 1] = presc_final[(size_t)i * n_steps + ST] - presc_init[(size_t)i * n_steps + ST];
        }
        Ubar0 = U;
        Uconv = U;
        double alpha_max = 1.0, alpha_min = 0.0, alpha = alpha_max, alpha_aux;
        int CutBack = 0;
        while (true) {
            const double Time = step_t0[ST] + alpha * step_dt[ST];
            for (int i = 0; i < n; ++i) {
                Fext[i] = Fext0[i] + alpha * dFext[i];
                Ubar[i] = Ubar0[i] + alpha * dUp[i];
            }
            // NewtonRaphsonFull_Solve (ModNewtonRaphsonFull.f90:44-168)
            X = Uconv;
            int it = 0;
            double normR0 = 0.0;
            bool ok = false;
            while (true) {
                // EvaluateR (ModFEMSystemOfEquations.f90:40-65)
                int nfail = 0;
                const int st = or_evaluate(m, Time, X.data(), fint.data(), kval.data(), &nfail, nullptr);
                if (st) break;
                for (int i = 0; i < n; ++i) R[i] = fint[i] - Fext[i];
                // EvaluateKt (:69-93): R = -R; ApplyBoundaryConditionsNEW; R = -R
                for (int i = 0; i < n; ++i) R[i] = -R[i];
                std::fill(Ud.begin(), Ud.end(), 0.0);
                if (n_presc) {
                    if (it == 0) {
                        for (int i = 0; i < n_presc; ++i) {
                            const int d = presc_dofs[i] - 1;
                            Ud[d] = Ubar[d] - X[d];
                        }
                        symv_upper(n, m->rowmap.data(), m->col.data(), kval.data(), Ud.data(), Rmod.data());
                        for (int i = 0; i < n; ++i) R[i] -= Rmod[i];
                    }
                    for (long long k : zp) kval[k] = 0.0;
                    for (long long k : op) kval[k] = 1.0;
                    for (int i = 0; i < n_presc; ++i) R[presc_dofs[i] - 1] = Ud[presc_dofs[i] - 1];
                }
                if (n_fixed) {
                    for (long long k : zf) kval[k] = 0.0;
                    for (long long k : of) kval[k] = 1.0;
                    for (int i = 0; i < n_fixed; ++i) R[fixed_dofs[i] - 1] = 0.0;
                }
                for (int i = 0; i < n; ++i) R[i] = -R[i];
                double normR = 0.0;
                if (norm_type == 2) {
                    for (int i = 0; i < n; ++i) normR = std::max(normR, std::fabs(R[i]));
                } else {
                    for (int i = 0; i < n; ++i) normR += R[i] * R[i];
                    normR = std::sqrt(normR);
                }
                if (nl < max_log) norm_log[nl] = normR;
                ++nl;
                if (it == 0) normR0 = normR;
                const double thr = norm_mode == 0 ? normR0 * tol : tol;
                if (it > 0 && normR < thr) { ok = true; break; }
                if (it >= itmax) break;
                ++it;
                Skyline sk;
                sk.build(n, m->rowmap.data(), m->col.data(), kval.data());
                if (!sk.factor()) break;
                for (int i = 0; i < n; ++i) DX[i] = -R[i];
                sk.solve(DX.data());
                for (int i = 0; i < n; ++i) X[i] += DX[i];
            }
            if (!ok) {
                alpha = alpha_min + (1.0 - 1.0 / GR) * (alpha - alpha_min);
                ++CutBack;
                if (CutBack > max_cutbacks) {
                    if (n_log) *n_log = nl;
                    return -1;
                }
                continue;
            }
            U = X;
            if (alpha == 1.0) {
                iters[ST] = it;
                cutbacks[ST] = CutBack;
                break;
            }
            alpha_aux = alpha_min;
            alpha_min = alpha;
            alpha = std::min(alpha + GR * (alpha - alpha_aux), 1.0);
            Uconv = U;
        }
        // SwitchConvergedState; the time of the converged step becomes the old time
        or_commit(m);
        m->time_old = step_t0[ST] + step_dt[ST];
        for (int p = 0; p < n_probe; ++p) probe_out[(size_t)p * n_steps + ST] = U[probe_dofs[p] - 1];
    }
    if (n_log) *n_log = nl;
    if (U_final) std::copy(U.begin(), U.end(), U_final);
    return 0;
}
