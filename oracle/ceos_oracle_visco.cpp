// ceos_oracle_visco.cpp -- TEST INFRASTRUCTURE ONLY.
//
// FP64 restatement of the reference's variational finite-strain viscoelastic model
// (ConstitutiveLibrary/ConstitutiveModelsLibrary/ModViscoelasticMatrix.f90): Neo-Hookean
// equilibrium branch plus one Maxwell branch F = Fe Fv with the viscous incompressibility
// J_v = 1 enforced by a Lagrange multiplier gamma, solved per Gauss point by a 7x7 local Newton
// (max 10 iterations, tolerance 1e-5), with the consistent tangent from the sensitivity of the
// local solution, pushed forward to the spatial Voigt modulus.
//
// Full (non-symmetric) second-order tensors use the reference's 9-component mapping of
// Tools/MathTools/ModVoigtNotation.f90 (component (i,j) at position i + 3 j, 0-based);
// fourth-order tensors are 9x9 matrices in that mapping.  All helpers below restate the
// semantics of the routines named in their comments.
#include <array>
#include <cmath>
#include <cstring>

namespace {

typedef std::array<double, 9> V9;
typedef std::array<double, 81> M9;  // row-major [p*9+q]

inline int vi(int i, int j) { return i + 3 * j; }

V9 eye9() { V9 a{}; a[0] = a[4] = a[8] = 1.0; return a; }
// DeterminantT2Voigt
double det9(const V9& a) {
    return a[0] * a[4] * a[8] - a[0] * a[7] * a[5] + a[1] * a[5] * a[6] - a[1] * a[3] * a[8] + a[2] * a[3] * a[7] -
           a[2] * a[4] * a[6];
}
// TransposeT2Voigt
V9 tr9(const V9& a) {
    V9 t;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[vi(i, j)] = a[vi(j, i)];
    return t;
}
// InverseT2Voigt: adjugate / determinant
V9 inv9(const V9& a) {
    V9 b;
    b[0] = a[4] * a[8] - a[7] * a[5];
    b[1] = a[2] * a[7] - a[1] * a[8];
    b[2] = -a[2] * a[4] + a[1] * a[5];
    b[3] = a[5] * a[6] - a[3] * a[8];
    b[4] = -a[2] * a[6] + a[0] * a[8];
    b[5] = a[2] * a[3] - a[0] * a[5];
    b[6] = a[3] * a[7] - a[4] * a[6];
    b[7] = a[1] * a[6] - a[0] * a[7];
    b[8] = -a[1] * a[3] + a[0] * a[4];
    const double d = det9(a);
    for (double& x : b) x /= d;
    return b;
}
// SingleContractionT2T2Voigt: matrix product A B
V9 mul9(const V9& a, const V9& b) {
    V9 c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[vi(i, k)] * b[vi(k, j)];
            c[vi(i, j)] = s;
        }
    return c;
}
V9 add(const V9& a, const V9& b, double sb = 1.0) { V9 c; for (int k = 0; k < 9; ++k) c[k] = a[k] + sb * b[k]; return c; }
V9 scale(const V9& a, double s) { V9 c; for (int k = 0; k < 9; ++k) c[k] = s * a[k]; return c; }
M9 madd(const M9& a, const M9& b, double sb = 1.0) { M9 c; for (int k = 0; k < 81; ++k) c[k] = a[k] + sb * b[k]; return c; }
M9 mscale(const M9& a, double s) { M9 c; for (int k = 0; k < 81; ++k) c[k] = s * a[k]; return c; }
// BallVoigt: (A (x) B)_ijkl = A_ij B_kl
M9 ball9(const V9& a, const V9& b) { M9 c; for (int p = 0; p < 9; ++p) for (int q = 0; q < 9; ++q) c[p * 9 + q] = a[p] * b[q]; return c; }
// SquareVoigt: (A [] B)_ijkl = A_ik B_jl
M9 square9(const V9& a, const V9& b) {
    M9 c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) c[vi(i, j) * 9 + vi(k, l)] = a[vi(i, k)] * b[vi(j, l)];
    return c;
}
// DoubleContractionT4T4Voigt: 9x9 product
M9 dc9(const M9& a, const M9& b) {
    M9 c;
    for (int p = 0; p < 9; ++p)
        for (int q = 0; q < 9; ++q) {
            double s = 0.0;
            for (int r = 0; r < 9; ++r) s += a[p * 9 + r] * b[r * 9 + q];
            c[p * 9 + q] = s;
        }
    return c;
}
inline int tp(int p) { return (p % 3) * 3 + p / 3; }  // index of the transposed pair
// RightSymmetrizationT4Voigt: A : Isym
M9 rsym(const M9& a) { M9 c; for (int p = 0; p < 9; ++p) for (int q = 0; q < 9; ++q) c[p * 9 + q] = 0.5 * (a[p * 9 + q] + a[p * 9 + tp(q)]); return c; }
// LeftSymmetrizationT4Voigt: Isym : A
M9 lsym(const M9& a) { M9 c; for (int p = 0; p < 9; ++p) for (int q = 0; q < 9; ++q) c[p * 9 + q] = 0.5 * (a[p * 9 + q] + a[tp(p) * 9 + q]); return c; }
// RigthLeftSymmetrizationT4Voigt: Isym : A : Isym
M9 rlsym(const M9& a) { return lsym(rsym(a)); }
// IdentityT4SymVoigt
M9 isym9() {
    M9 c{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l)
                    c[vi(i, j) * 9 + vi(k, l)] = 0.5 * ((i == k && j == l ? 1.0 : 0.0) + (i == l && j == k ? 1.0 : 0.0));
    return c;
}
// Tensor2VoigtToTensor2VoigtSym: (A11, A22, A33, A12, A23, A31)
void to_sym6(const V9& a, double s[6]) { s[0] = a[0]; s[1] = a[4]; s[2] = a[8]; s[3] = a[3]; s[4] = a[7]; s[5] = a[2]; }
// Tensor2VoigtSymToTensor2Voigt
V9 from_sym6(const double s[6]) { return V9{s[0], s[3], s[5], s[3], s[1], s[4], s[5], s[4], s[2]}; }
// Tensor4VoigtToTensor4VoigtSym: rows/columns 11, 22, 33, 12, 23, 13
const int kSymMap[6] = {0, 4, 8, 3, 7, 6};
void t4sym(const M9& a, double t[6][6]) { for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) t[r][c] = a[kSymMap[r] * 9 + kSymMap[c]]; }

// dgetrf + dgetrs: Gaussian elimination with partial pivoting, n x n, nrhs right-hand sides
// (column-major B [n][nrhs] stored as b[i*nrhs + c]).
bool lu_solve(int n, double* A, double* b, int nrhs) {
    int piv[16];
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i) if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
        piv[k] = p;
        if (A[p * n + k] == 0.0) return false;
        if (p != k) for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
        for (int i = k + 1; i < n; ++i) {
            A[i * n + k] /= A[k * n + k];
            for (int j = k + 1; j < n; ++j) A[i * n + j] -= A[i * n + k] * A[k * n + j];
        }
    }
    for (int c = 0; c < nrhs; ++c) {
        for (int k = 0; k < n; ++k) if (piv[k] != k) std::swap(b[k * nrhs + c], b[piv[k] * nrhs + c]);
        for (int i = 1; i < n; ++i) for (int j = 0; j < i; ++j) b[i * nrhs + c] -= A[i * n + j] * b[j * nrhs + c];
        for (int i = n - 1; i >= 0; --i) {
            for (int j = i + 1; j < n; ++j) b[i * nrhs + c] -= A[i * n + j] * b[j * nrhs + c];
            b[i * nrhs + c] /= A[i * n + i];
        }
    }
    return true;
}

struct Branch {  // quantities of one local-Newton iterate (Local_Newton_Raphson_MATRIX)
    V9 Fv, FvFvoi, Ce, Se, Me;
    M9 De;
    double Jv;
};

Branch branch_state(const V9& F, const V9& Fv_old, const V9& dv, double dt, double Mu_e) {
    Branch s;
    const V9 I = eye9();
    s.Fv = mul9(inv9(add(I, dv, -dt)), Fv_old);
    s.Jv = det9(s.Fv);
    s.FvFvoi = mul9(s.Fv, inv9(Fv_old));
    const V9 Fe = mul9(F, inv9(s.Fv));
    s.Ce = mul9(tr9(Fe), Fe);
    const V9 Cei = inv9(s.Ce);
    s.Se = scale(add(I, Cei, -1.0), Mu_e);
    s.De = mscale(rsym(square9(Cei, Cei)), 2.0 * Mu_e);
    s.Me = mul9(s.Ce, s.Se);
    return s;
}

// Residual_MATRIX (:573-623)
void residual(const Branch& s, double gama, const V9& dv, double Ni_v, double dt, double Rm[7]) {
    V9 DP = scale(mul9(tr9(s.FvFvoi), s.Me), -dt);
    DP = scale(add(DP, tr9(DP)), 0.5);
    DP = add(DP, scale(dv, Ni_v), dt);
    const V9 DJ = scale(s.FvFvoi, dt * s.Jv);
    const V9 DL = add(DP, DJ, gama);
    to_sym6(DL, Rm);
    Rm[6] = s.Jv - 1.0;
}

// Jacobian_MATRIX (:627-734): Km (7x7) and DSem_Ddvm
void jacobian(const Branch& s, const V9& Fv_old, double gama, double Ni_v, double dt, double Km[7][7], M9& DSe_Ddv) {
    const V9 I = eye9();
    const M9 B = square9(mul9(s.Ce, s.FvFvoi), I);
    const M9 DCe_Ddv = mscale(rlsym(B), -2.0 * dt);
    DSe_Ddv = mscale(rsym(dc9(s.De, B)), -dt);
    const M9 DMe_Ddv = madd(dc9(square9(I, s.Se), DCe_Ddv), dc9(square9(s.Ce, I), DSe_Ddv));
    const V9 Aux1 = mul9(tr9(inv9(Fv_old)), s.FvFvoi);
    const V9 Aux2 = tr9(mul9(s.Fv, s.Me));
    M9 D2He = madd(mscale(square9(Aux1, Aux2), dt * dt), mscale(dc9(square9(tr9(s.FvFvoi), I), DMe_Ddv), dt));
    D2He = mscale(rlsym(D2He), -1.0);
    const M9 D2Pinc = madd(D2He, mscale(isym9(), Ni_v * dt));
    const M9 D2Jv = mscale(rlsym(madd(ball9(s.FvFvoi, s.FvFvoi), square9(s.FvFvoi, s.FvFvoi))), dt * dt * s.Jv);
    const M9 D2L = madd(D2Pinc, D2Jv, gama);
    const V9 D2Lg = scale(s.FvFvoi, dt * s.Jv);
    double t[6][6], a[6];
    t4sym(D2L, t);
    to_sym6(D2Lg, a);
    for (int r = 0; r < 7; ++r) for (int c = 0; c < 7; ++c) Km[r][c] = 0.0;
    for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) Km[r][c] = t[r][c];
    for (int j = 0; j < 6; ++j) { Km[j][6] = a[j]; Km[6][j] = a[j]; }
    // correction for the symmetric Voigt mapping: right-multiply by diag(1,1,1,2,2,2)
    for (int r = 0; r < 7; ++r) for (int c = 3; c < 6; ++c) Km[r][c] *= 2.0;
}

}  // namespace

// params [K_inf, Mu_inf, Lambda_inf, K_e, Mu_e, Ni_v]; state [Fv (9), dv (9), gamma]
int visco_var_update(const double* p, const double* Fin, double dt, const double* st_old, double* st_new,
                     double* sig, double* D) {
    const double Mu_inf = p[1], Lambda_inf = p[2], Mu_e = p[4], Ni_v = p[5];
    V9 F;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) F[vi(i, j)] = Fin[i * 3 + j];  // Tensor2ToVoigt
    V9 Fv_old;
    for (int k = 0; k < 9; ++k) Fv_old[k] = st_old[k];
    const double gama_old = st_old[18];
    const V9 I = eye9();
    // ---- Local_Newton_Raphson_MATRIX (:408-569) ----
    double X[7];
    V9 dv{};
    double gama = gama_old;
    to_sym6(dv, X);
    X[6] = gama;
    Branch s;
    int status = 2;
    for (int it = 1; it <= 10; ++it) {
        s = branch_state(F, Fv_old, dv, dt, Mu_e);
        double Rm[7];
        residual(s, gama, dv, Ni_v, dt, Rm);
        double nr = 0.0;
        for (double r : Rm) nr += r * r;
        if (std::sqrt(nr) < 1.0e-5) { status = 0; break; }
        double Km[7][7];
        M9 DSe;
        jacobian(s, Fv_old, gama, Ni_v, dt, Km, DSe);
        double b[7];
        for (int k = 0; k < 7; ++k) b[k] = -Rm[k];
        if (!lu_solve(7, &Km[0][0], b, 1)) break;
        for (int k = 0; k < 7; ++k) X[k] += b[k];
        dv = from_sym6(X);
        gama = X[6];
    }
    // new state (the reference stores the last iterate; Fv from the converged iterate)
    for (int k = 0; k < 9; ++k) { st_new[k] = s.Fv[k]; st_new[9 + k] = dv[k]; }
    st_new[18] = gama;
    // ---- stress (UpdateStressAndStateVariables_ViscoelasticMatrix_3D :276-402) ----
    const double J = det9(F);
    const V9 C = mul9(tr9(F), F);
    const V9 Ci = inv9(C);
    const V9 Sinf = add(scale(add(I, Ci, -1.0), Mu_inf), scale(Ci, Lambda_inf * std::log(J)));
    const V9 Fvi = inv9(s.Fv);
    const V9 Sm = add(Sinf, mul9(mul9(Fvi, s.Se), tr9(Fvi)));
    const V9 cau = scale(mul9(mul9(F, Sm), tr9(F)), 1.0 / J);  // StressTransformation, PK2 -> Cauchy
    sig[0] = cau[vi(0, 0)]; sig[1] = cau[vi(1, 1)]; sig[2] = cau[vi(2, 2)];
    sig[3] = cau[vi(0, 1)]; sig[4] = cau[vi(1, 2)]; sig[5] = cau[vi(0, 2)];
    // ---- tangent (GetTangentModulus_ViscoelasticMatrix_3D :745-998) ----
    const Branch t = branch_state(F, Fv_old, dv, dt, Mu_e);  // Fv recomputed from dv_new
    const V9 Fvn_i = inv9(t.Fv);
    const M9 FviSq = square9(Fvn_i, Fvn_i);
    const M9 FviTSq = square9(tr9(Fvn_i), tr9(Fvn_i));
    const M9 Dinf = madd(mscale(ball9(Ci, Ci), Lambda_inf),
                         mscale(rsym(square9(Ci, Ci)), 2.0 * (Mu_inf - Lambda_inf * std::log(J))));
    double Km[7][7];
    M9 DSe_Ddv;
    jacobian(t, Fv_old, gama, Ni_v, dt, Km, DSe_Ddv);
    const M9 W = dc9(dc9(FviSq, t.De), FviTSq);
    const M9 DS_DC = mscale(madd(Dinf, rlsym(W)), 0.5);
    M9 Z = mscale(square9(inv9(Fv_old), mul9(Fvn_i, t.Se)), -2.0 * dt);
    Z = madd(Z, dc9(FviSq, DSe_Ddv));
    const M9 DS_Ddv = rlsym(Z);
    const M9 DCe_DC = rsym(FviTSq);
    const M9 DSe_DC = mscale(dc9(t.De, DCe_DC), 0.5);
    const M9 DMe_DC = madd(dc9(square9(I, t.Se), DCe_DC), dc9(square9(t.Ce, I), DSe_DC));
    const M9 G = dc9(square9(tr9(t.FvFvoi), I), DMe_DC);
    const M9 D2L_DCDdv = mscale(rlsym(G), -dt);
    double drm[6][6];
    t4sym(D2L_DCDdv, drm);
    double rhs[7 * 6];  // -Drm_DC, 7 x 6 (row 7 zero)
    for (int r = 0; r < 7; ++r) for (int c = 0; c < 6; ++c) rhs[r * 6 + c] = r < 6 ? -drm[r][c] : 0.0;
    double Kc[49];
    std::memcpy(Kc, &Km[0][0], sizeof(Kc));
    if (!lu_solve(7, Kc, rhs, 6)) status = 2;
    double sdv[6][6], sdc[6][6], Dm[6][6];
    t4sym(DS_Ddv, sdv);
    t4sym(DS_DC, sdc);
    // DoubleContractionT4T4VoigtSym(sdv, ddv_dC): sdv * (ddv_dC with rows 4..6 doubled)
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += sdv[r][k] * rhs[k * 6 + c] * (k >= 3 ? 2.0 : 1.0);
            Dm[r][c] = 2.0 * (sdc[r][c] + acc);
        }
    // Push_Forward_Voigt (ModMathRoutines.f90:254-311): A Dm A^T / J, Dm read through its upper triangle
    double Ft[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Ft[i][j] = Fin[j * 3 + i];
    double A[6][6];
    const int P[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 2}, {0, 2}};
    for (int r = 0; r < 6; ++r) {
        const int a = P[r][0], b = P[r][1];
        for (int c = 0; c < 6; ++c) {
            const int k = P[c][0], l = P[c][1];
            // row r of A maps a material symmetric component to spatial (a,b): F_ak F_bl (+ sym)
            if (c < 3) A[r][c] = Ft[k][a] * Ft[k][b];
            else A[r][c] = Ft[k][a] * Ft[l][b] + Ft[l][a] * Ft[k][b];
        }
    }
    double Ws[6][6], AW[6][6];
    for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) Ws[r][c] = r <= c ? Dm[r][c] : Dm[c][r];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += A[r][k] * Ws[k][c];
            AW[r][c] = acc;
        }
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += AW[r][k] * A[c][k];
            D[r * 6 + c] = acc / J;
        }
    return status;
}
