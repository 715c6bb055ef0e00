// visco_var.cuh -- the reference's variational viscoelastic model on the device.
//
// ConstitutiveModelsLibrary/ModViscoelasticMatrix.f90: Neo-Hookean equilibrium branch (Mu_inf,
// Lambda_inf) plus one Maxwell branch F = Fe Fv with a Neo-Hookean elastic part (Mu_e), quadratic
// viscous potential (Ni_v) and J_v = 1 enforced through the multiplier gamma.  Per Gauss point:
// a 7x7 local Newton on (d_v sym, gamma) (Local_Newton_Raphson_MATRIX :408-569, max 10
// iterations, tolerance 1e-5 on the residual norm), the stress (:276-402), and the consistent
// tangent from the sensitivity of the local solution (GetTangentModulus :745-998) pushed
// forward with Push_Forward_Voigt (ModMathRoutines.f90:254-311).
//
// Everything is evaluated in FP64 (the local Newton needs it) whatever the element type.
// Full second-order tensors use the reference's 9-component layout (component (i,j) at i+3j,
// ModVoigtNotation.f90:70-105); fourth-order tensors are row-major 9x9 arrays in that layout.
#pragma once
#include "ceos_common.cuh"

namespace ceos {
namespace vv {

struct T2 { double v[9]; };
struct T4 { double v[81]; };

CEOS_HD int id9(int i, int j) { return i + 3 * j; }
CEOS_HD int tidx(int p) { return (p % 3) * 3 + p / 3; }

CEOS_D T2 eye() { T2 a; for (int k = 0; k < 9; ++k) a.v[k] = (k == 0 || k == 4 || k == 8) ? 1.0 : 0.0; return a; }
CEOS_D double det(const T2& a) {
    const double* x = a.v;
    return x[0] * x[4] * x[8] - x[0] * x[7] * x[5] + x[1] * x[5] * x[6] - x[1] * x[3] * x[8] + x[2] * x[3] * x[7] -
           x[2] * x[4] * x[6];
}
CEOS_D T2 tr(const T2& a) { T2 t; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.v[id9(i, j)] = a.v[id9(j, i)]; return t; }
CEOS_D T2 inv(const T2& a) {
    const double* x = a.v;
    T2 b;
    b.v[0] = x[4] * x[8] - x[7] * x[5];
    b.v[1] = x[2] * x[7] - x[1] * x[8];
    b.v[2] = -x[2] * x[4] + x[1] * x[5];
    b.v[3] = x[5] * x[6] - x[3] * x[8];
    b.v[4] = -x[2] * x[6] + x[0] * x[8];
    b.v[5] = x[2] * x[3] - x[0] * x[5];
    b.v[6] = x[3] * x[7] - x[4] * x[6];
    b.v[7] = x[1] * x[6] - x[0] * x[7];
    b.v[8] = -x[1] * x[3] + x[0] * x[4];
    const double r = 1.0 / det(a);
    for (int k = 0; k < 9; ++k) b.v[k] *= r;
    return b;
}
CEOS_D T2 mul(const T2& a, const T2& b) {
    T2 c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            c.v[id9(i, j)] = a.v[id9(i, 0)] * b.v[id9(0, j)] + a.v[id9(i, 1)] * b.v[id9(1, j)] + a.v[id9(i, 2)] * b.v[id9(2, j)];
    return c;
}
CEOS_D T2 axpy(const T2& a, double s, const T2& b) { T2 c; for (int k = 0; k < 9; ++k) c.v[k] = a.v[k] + s * b.v[k]; return c; }
CEOS_D T2 scal(double s, const T2& a) { T2 c; for (int k = 0; k < 9; ++k) c.v[k] = s * a.v[k]; return c; }
// (A [] B)_ijkl = A_ik B_jl  (SquareVoigt)
CEOS_D void square(const T2& a, const T2& b, T4& c) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) c.v[id9(i, j) * 9 + id9(k, l)] = a.v[id9(i, k)] * b.v[id9(j, l)];
}
// C = A B (DoubleContractionT4T4Voigt); C may not alias A or B
CEOS_D void dc(const T4& a, const T4& b, T4& c) {
    for (int p = 0; p < 9; ++p)
        for (int q = 0; q < 9; ++q) {
            double s = 0.0;
            for (int r = 0; r < 9; ++r) s += a.v[p * 9 + r] * b.v[r * 9 + q];
            c.v[p * 9 + q] = s;
        }
}
// in-place Isym : A : Isym (RigthLeftSymmetrizationT4Voigt) and A : Isym (RightSymmetrizationT4Voigt)
CEOS_D void rlsym(T4& a) {
    for (int p = 0; p < 9; ++p)
        for (int q = 0; q < 9; ++q) {
            const int pt = tidx(p), qt = tidx(q);
            if (p * 9 + q > pt * 9 + qt) continue;  // handle each orbit {(p,q),(pt,qt),(p,qt),(pt,q)} once
            if (p * 9 + q > p * 9 + qt || p * 9 + q > pt * 9 + q) continue;
            const double m = 0.25 * (a.v[p * 9 + q] + a.v[p * 9 + qt] + a.v[pt * 9 + q] + a.v[pt * 9 + qt]);
            a.v[p * 9 + q] = a.v[p * 9 + qt] = a.v[pt * 9 + q] = a.v[pt * 9 + qt] = m;
        }
}
CEOS_D void rsym(T4& a) {
    for (int p = 0; p < 9; ++p)
        for (int q = 0; q < 9; ++q) {
            const int qt = tidx(q);
            if (q >= qt) continue;
            const double m = 0.5 * (a.v[p * 9 + q] + a.v[p * 9 + qt]);
            a.v[p * 9 + q] = a.v[p * 9 + qt] = m;
        }
}
CEOS_D void sym6(const T2& a, double s[6]) { s[0] = a.v[0]; s[1] = a.v[4]; s[2] = a.v[8]; s[3] = a.v[3]; s[4] = a.v[7]; s[5] = a.v[2]; }
CEOS_D T2 unsym6(const double s[6]) {
    T2 a;
    a.v[0] = s[0]; a.v[1] = s[3]; a.v[2] = s[5]; a.v[3] = s[3]; a.v[4] = s[1];
    a.v[5] = s[4]; a.v[6] = s[5]; a.v[7] = s[4]; a.v[8] = s[2];
    return a;
}
CEOS_HD int smap(int r) { return r == 0 ? 0 : r == 1 ? 4 : r == 2 ? 8 : r == 3 ? 3 : r == 4 ? 7 : 6; }

// LU with partial pivoting (dgetrf/dgetrs), n = 7, nrhs right-hand sides stored b[i*nrhs+c]
CEOS_D bool lu7(double* A, double* b, int nrhs) {
    int piv[7];
    for (int k = 0; k < 7; ++k) {
        int p = k;
        for (int i = k + 1; i < 7; ++i) if (fabs(A[i * 7 + k]) > fabs(A[p * 7 + k])) p = i;
        piv[k] = p;
        if (A[p * 7 + k] == 0.0) return false;
        if (p != k) for (int j = 0; j < 7; ++j) { const double t = A[k * 7 + j]; A[k * 7 + j] = A[p * 7 + j]; A[p * 7 + j] = t; }
        const double rk = 1.0 / A[k * 7 + k];
        for (int i = k + 1; i < 7; ++i) {
            A[i * 7 + k] *= rk;
            for (int j = k + 1; j < 7; ++j) A[i * 7 + j] -= A[i * 7 + k] * A[k * 7 + j];
        }
    }
    for (int c = 0; c < nrhs; ++c) {
        for (int k = 0; k < 7; ++k)
            if (piv[k] != k) { const double t = b[k * nrhs + c]; b[k * nrhs + c] = b[piv[k] * nrhs + c]; b[piv[k] * nrhs + c] = t; }
        for (int i = 1; i < 7; ++i) for (int j = 0; j < i; ++j) b[i * nrhs + c] -= A[i * 7 + j] * b[j * nrhs + c];
        for (int i = 6; i >= 0; --i) {
            for (int j = i + 1; j < 7; ++j) b[i * nrhs + c] -= A[i * 7 + j] * b[j * nrhs + c];
            b[i * nrhs + c] /= A[i * 7 + i];
        }
    }
    return true;
}

struct Iterate { T2 Fv, FvFvoi, Ce, Se, Me, Cei; double Jv; };

CEOS_D void iterate(const T2& F, const T2& Fv_old, const T2& Fvoi, const T2& dv, double dt, double Mu_e, Iterate& s) {
    const T2 I = eye();
    s.Fv = mul(inv(axpy(I, -dt, dv)), Fv_old);
    s.Jv = det(s.Fv);
    s.FvFvoi = mul(s.Fv, Fvoi);
    const T2 Fe = mul(F, inv(s.Fv));
    s.Ce = mul(tr(Fe), Fe);
    s.Cei = inv(s.Ce);
    s.Se = scal(Mu_e, axpy(I, -1.0, s.Cei));
    s.Me = mul(s.Ce, s.Se);
}

// De = 2 Mu_e (Cei [] Cei) : Isym
CEOS_D void elastic_modulus(const Iterate& s, double Mu_e, T4& De) {
    square(s.Cei, s.Cei, De);
    rsym(De);
    for (int k = 0; k < 81; ++k) De.v[k] *= 2.0 * Mu_e;
}

// Jacobian_MATRIX (ModViscoelasticMatrix.f90:627-734): Km and DSe_Ddv.  w1, w2 are work arrays.
CEOS_D void jacobian(const Iterate& s, const T4& De, const T2& Fvoi, double gama, double Ni_v, double dt, double Km[49],
                     T4& DSe_Ddv, T4& w1, T4& w2, T4& w3) {
    const T2 I = eye();
    // B = (Ce FvFvoi) [] I
    square(mul(s.Ce, s.FvFvoi), I, w1);                       // w1 = B
    dc(De, w1, DSe_Ddv);                                      // DSe_Ddv = -dt (De : B) : Isym
    rsym(DSe_Ddv);
    for (int k = 0; k < 81; ++k) DSe_Ddv.v[k] *= -dt;
    rlsym(w1);                                                // w1 = DCe_Ddv / (-2 dt)
    for (int k = 0; k < 81; ++k) w1.v[k] *= -2.0 * dt;
    square(I, s.Se, w2);                                      // DMe_Ddv = (I [] Se) DCe + (Ce [] I) DSe
    dc(w2, w1, w3);
    square(s.Ce, I, w2);
    dc(w2, DSe_Ddv, w1);
    for (int k = 0; k < 81; ++k) w3.v[k] += w1.v[k];          // w3 = DMe_Ddv
    square(tr(s.FvFvoi), I, w2);
    dc(w2, w3, w1);                                           // w1 = (FvFvoi^T [] I) DMe
    const T2 Aux1 = mul(tr(Fvoi), s.FvFvoi);
    const T2 Aux2 = tr(mul(s.Fv, s.Me));
    square(Aux1, Aux2, w2);
    for (int k = 0; k < 81; ++k) w2.v[k] = dt * dt * w2.v[k] + dt * w1.v[k];  // D2He before symmetrization
    rlsym(w2);
    // D2L = -D2He + dt Ni_v Isym + gama dt^2 Jv Isym:(FvFvoi (x) FvFvoi + FvFvoi [] FvFvoi):Isym
    square(s.FvFvoi, s.FvFvoi, w1);
    for (int p = 0; p < 9; ++p)
        for (int q = 0; q < 9; ++q) w1.v[p * 9 + q] += s.FvFvoi.v[p] * s.FvFvoi.v[q];
    rlsym(w1);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) {
                    const int p = id9(i, j) * 9 + id9(k, l);
                    const double isym = 0.5 * ((i == k && j == l ? 1.0 : 0.0) + (i == l && j == k ? 1.0 : 0.0));
                    w2.v[p] = -w2.v[p] + dt * Ni_v * isym + gama * dt * dt * s.Jv * w1.v[p];
                }
    double a[6];
    sym6(scal(dt * s.Jv, s.FvFvoi), a);
    for (int r = 0; r < 7; ++r)
        for (int c = 0; c < 7; ++c) {
            double v;
            if (r < 6 && c < 6) v = w2.v[smap(r) * 9 + smap(c)];
            else if (r < 6) v = a[r];
            else if (c < 6) v = a[c];
            else v = 0.0;
            Km[r * 7 + c] = (c >= 3 && c < 6) ? 2.0 * v : v;  // symmetric-Voigt correction (IdentityT4SymInv)
        }
}

// One Gauss point.  st: [Fv (9), dv (9), gamma]; returns 0 or 2 (local Newton not converged).
// sig: Cauchy (Voigt 6); D: spatial tangent, upper 21.
template <typename T>
CEOS_D int update(const T Fin[3][3], const T* p, double dt, const T* st, T* stn, T sig[6], T D[21]) {
    const double Mu_inf = p[1], Lambda_inf = p[2], Mu_e = p[4], Ni_v = p[5];
    T2 F, Fv_old;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) F.v[id9(i, j)] = (double)Fin[i][j];
    for (int k = 0; k < 9; ++k) Fv_old.v[k] = (double)st[k];
    const double gama_old = (double)st[18];
    const T2 I = eye();
    const T2 Fvoi = inv(Fv_old);
    T4 De, DSe, w1, w2, w3;
    double X[7];
    T2 dv;
    for (int k = 0; k < 9; ++k) dv.v[k] = 0.0;
    double gama = gama_old;
    sym6(dv, X);
    X[6] = gama;
    Iterate s;
    int status = 2;
    for (int it = 0; it < 10; ++it) {
        iterate(F, Fv_old, Fvoi, dv, dt, Mu_e, s);
        // Residual_MATRIX (:573-623)
        T2 DP = scal(-dt, mul(tr(s.FvFvoi), s.Me));
        DP = scal(0.5, axpy(DP, 1.0, tr(DP)));
        DP = axpy(DP, dt * Ni_v, dv);
        const T2 DL = axpy(DP, gama * dt * s.Jv, s.FvFvoi);
        double Rm[7];
        sym6(DL, Rm);
        Rm[6] = s.Jv - 1.0;
        double nr = 0.0;
        for (int k = 0; k < 7; ++k) nr += Rm[k] * Rm[k];
        if (sqrt(nr) < 1.0e-5) { status = 0; break; }
        elastic_modulus(s, Mu_e, De);
        double Km[49];
        jacobian(s, De, Fvoi, gama, Ni_v, dt, Km, DSe, w1, w2, w3);
        for (int k = 0; k < 7; ++k) Rm[k] = -Rm[k];
        if (!lu7(Km, Rm, 1)) break;
        for (int k = 0; k < 7; ++k) X[k] += Rm[k];
        dv = unsym6(X);
        gama = X[6];
    }
    for (int k = 0; k < 9; ++k) { stn[k] = (T)s.Fv.v[k]; stn[9 + k] = (T)dv.v[k]; }
    stn[18] = (T)gama;
    // stress
    const double J = det(F);
    const double lnJ = log(J);
    const T2 Ci = inv(mul(tr(F), F));
    const T2 Fvi = inv(s.Fv);
    T2 Sm = axpy(scal(Mu_inf, axpy(I, -1.0, Ci)), Lambda_inf * lnJ, Ci);
    Sm = axpy(Sm, 1.0, mul(mul(Fvi, s.Se), tr(Fvi)));
    const T2 cau = scal(1.0 / J, mul(mul(F, Sm), tr(F)));
    sig[0] = (T)cau.v[0]; sig[1] = (T)cau.v[4]; sig[2] = (T)cau.v[8];
    sig[3] = (T)cau.v[3]; sig[4] = (T)cau.v[7]; sig[5] = (T)cau.v[6];
    // tangent: recompute the branch from dv_new (GetTangentModulus :829-971)
    iterate(F, Fv_old, Fvoi, dv, dt, Mu_e, s);
    elastic_modulus(s, Mu_e, De);
    double Km[49];
    jacobian(s, De, Fvoi, gama, Ni_v, dt, Km, DSe, w1, w2, w3);
    const T2 Fvn_i = inv(s.Fv);
    // DS_Ddv = Isym:( -2 dt Fv_old^-1 [] (Fv^-1 Se) + (Fv^-1 [] Fv^-1) DSe_Ddv ):Isym   -> w3
    square(Fvn_i, Fvn_i, w1);
    dc(w1, DSe, w3);
    square(Fvoi, mul(Fvn_i, s.Se), w2);
    for (int k = 0; k < 81; ++k) w3.v[k] += -2.0 * dt * w2.v[k];
    rlsym(w3);
    double sdv[36];
    for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) sdv[r * 6 + c] = w3.v[smap(r) * 9 + smap(c)];
    // DCe_DC = (Fv^-T [] Fv^-T):Isym -> w2 ; DSe_DC = 1/2 De DCe_DC -> w3
    const T2 FviT = tr(Fvn_i);
    square(FviT, FviT, w2);
    rsym(w2);
    dc(De, w2, w3);
    for (int k = 0; k < 81; ++k) w3.v[k] *= 0.5;
    // DMe_DC = (I [] Se) DCe_DC + (Ce [] I) DSe_DC -> DSe (reused)
    square(I, s.Se, w1);
    dc(w1, w2, DSe);
    square(s.Ce, I, w1);
    dc(w1, w3, w2);
    for (int k = 0; k < 81; ++k) DSe.v[k] += w2.v[k];
    // D2L_DCDdv = -dt Isym:((FvFvoi^T [] I) DMe_DC):Isym -> w1
    square(tr(s.FvFvoi), I, w2);
    dc(w2, DSe, w1);
    rlsym(w1);
    double rhs[42];
    for (int r = 0; r < 7; ++r)
        for (int c = 0; c < 6; ++c) rhs[r * 6 + c] = r < 6 ? dt * w1.v[smap(r) * 9 + smap(c)] : 0.0;  // -Drm_DC
    int st2 = lu7(Km, rhs, 6) ? 0 : 2;
    // DS_DC = 1/2 (Dinf + Isym:((Fv^-1 [] Fv^-1) De (Fv^-T [] Fv^-T)):Isym) -> w3
    square(Fvn_i, Fvn_i, w1);
    dc(w1, De, w2);
    square(FviT, FviT, w1);
    dc(w2, w1, w3);
    rlsym(w3);
    square(Ci, Ci, w1);
    rsym(w1);
    for (int pq = 0; pq < 81; ++pq) {
        const double dinf = Lambda_inf * Ci.v[pq / 9] * Ci.v[pq % 9] + 2.0 * (Mu_inf - Lambda_inf * lnJ) * w1.v[pq];
        w3.v[pq] = 0.5 * (dinf + w3.v[pq]);
    }
    double Dm[36];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += sdv[r * 6 + k] * rhs[k * 6 + c] * (k >= 3 ? 2.0 : 1.0);
            Dm[r * 6 + c] = 2.0 * (w3.v[smap(r) * 9 + smap(c)] + acc);
        }
    // push-forward: D = A sym_upper(Dm) A^T / J
    double A[36];
    const int P0[6] = {0, 1, 2, 0, 1, 0}, P1[6] = {0, 1, 2, 1, 2, 2};
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            const int a = P0[r], b = P1[r], k = P0[c], l = P1[c];
            const double Fak = F.v[id9(a, k)], Fbl = F.v[id9(b, l)], Fal = F.v[id9(a, l)], Fbk = F.v[id9(b, k)];
            A[r * 6 + c] = c < 3 ? Fak * Fbk : Fak * Fbl + Fal * Fbk;
        }
    double AW[36];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += A[r * 6 + k] * (k <= c ? Dm[k * 6 + c] : Dm[c * 6 + k]);
            AW[r * 6 + c] = acc;
        }
    const double rJ = 1.0 / J;
    for (int r = 0; r < 6; ++r)
        for (int c = r; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += AW[r * 6 + k] * A[c * 6 + k];
            D[up21(r, c)] = (T)(acc * rJ);
        }
    return status ? status : st2;
}

}  // namespace vv
}  // namespace ceos
