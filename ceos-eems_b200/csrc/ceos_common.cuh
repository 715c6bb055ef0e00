// ceos_common.cuh -- shared device helpers for the sm_100a element loop.
//
// Symmetric second-order tensors are held in the reference's Voigt order
// 11, 22, 33, 12, 23, 13 (Convert_to_Voigt_3D_Sym, Tools/MathTools/ModMathRoutines.f90:660-674);
// 6x6 spatial tangents in the same order with tensorial shear (IsymV has 1/2 on the shear
// diagonal, ModMathRoutines.f90:194-207), so that sigma = D * strain with engineering shear.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CEOS_HD __host__ __device__ __forceinline__
#define CEOS_D __device__ __forceinline__

namespace ceos {

// Hexa8 local node signs (FEM/Elements/ElementLibrary/ModElementHexa8.f90:185-192).
constexpr int kSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                             {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// Index of the local node pair (i < j) in the 28-entry per-element rank table.
CEOS_HD int pair_index(int i, int j) { return 7 * i - (i * (i - 1)) / 2 + (j - i - 1); }

CEOS_HD constexpr double delta6(int k) { return k < 3 ? 1.0 : 0.0; }

template <typename T>
struct Sym6 {
    T v[6];
};

// det (Tools/MathTools/ModMathRoutines.f90:16-31), same term order, in FP64.
template <typename T>
CEOS_HD double det3_fp64(const T F[3][3]) {
    const double a00 = F[0][0], a01 = F[0][1], a02 = F[0][2], a10 = F[1][0], a11 = F[1][1], a12 = F[1][2],
                 a20 = F[2][0], a21 = F[2][1], a22 = F[2][2];
    return a00 * a11 * a22 + a01 * a12 * a20 + a02 * a10 * a21 - a02 * a11 * a20 - a01 * a10 * a22 - a00 * a12 * a21;
}

template <typename T>
CEOS_HD T det3(const T F[3][3]) {
    return F[0][0] * F[1][1] * F[2][2] + F[0][1] * F[1][2] * F[2][0] + F[0][2] * F[1][0] * F[2][1] -
           F[0][2] * F[1][1] * F[2][0] - F[0][1] * F[1][0] * F[2][2] - F[0][0] * F[1][2] * F[2][1];
}

// inverse (ModMathRoutines.f90:33-62): adjugate divided by the determinant.
template <typename T>
CEOS_HD void inv3(const T A[3][3], T d, T B[3][3]) {
    B[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    B[0][1] = A[0][2] * A[2][1] - A[0][1] * A[2][2];
    B[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
    B[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    B[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
    B[1][2] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
    B[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    B[2][1] = A[0][1] * A[2][0] - A[0][0] * A[2][1];
    B[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    const T r = T(1) / d;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) B[i][j] = B[i][j] * r;
}

// b = F F^T (Voigt)
template <typename T>
CEOS_HD void ffT(const T F[3][3], T b[6]) {
    const int I[6] = {0, 1, 2, 0, 1, 0}, J[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) b[k] = F[I[k]][0] * F[J[k]][0] + F[I[k]][1] * F[J[k]][1] + F[I[k]][2] * F[J[k]][2];
}
// C = F^T F (Voigt)
template <typename T>
CEOS_HD void fTf(const T F[3][3], T C[6]) {
    const int I[6] = {0, 1, 2, 0, 1, 0}, J[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) C[k] = F[0][I[k]] * F[0][J[k]] + F[1][I[k]] * F[1][J[k]] + F[2][I[k]] * F[2][J[k]];
}
template <typename T>
CEOS_HD void sym_to_mat(const T v[6], T A[3][3]) {
    A[0][0] = v[0]; A[1][1] = v[1]; A[2][2] = v[2];
    A[0][1] = A[1][0] = v[3];
    A[1][2] = A[2][1] = v[4];
    A[0][2] = A[2][0] = v[5];
}
// F S F^T for symmetric S (Voigt in, Voigt out)
template <typename T>
CEOS_HD void push_sym(const T F[3][3], const T S[6], T out[6]) {
    T Sm[3][3], Tm[3][3];
    sym_to_mat(S, Sm);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Tm[i][j] = Sm[i][0] * F[j][0] + Sm[i][1] * F[j][1] + Sm[i][2] * F[j][2];
    const int I[6] = {0, 1, 2, 0, 1, 0}, J[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = F[I[k]][0] * Tm[0][J[k]] + F[I[k]][1] * Tm[1][J[k]] + F[I[k]][2] * Tm[2][J[k]];
}
// inverse of a symmetric tensor in Voigt form, given its determinant
template <typename T>
CEOS_HD void inv_sym(const T c[6], T d, T ci[6]) {
    // c = [[c0 c3 c5],[c3 c1 c4],[c5 c4 c2]]
    const T r = T(1) / d;
    ci[0] = (c[1] * c[2] - c[4] * c[4]) * r;
    ci[1] = (c[0] * c[2] - c[5] * c[5]) * r;
    ci[2] = (c[0] * c[1] - c[3] * c[3]) * r;
    ci[3] = (c[5] * c[4] - c[3] * c[2]) * r;
    ci[4] = (c[3] * c[5] - c[0] * c[4]) * r;
    ci[5] = (c[3] * c[4] - c[5] * c[1]) * r;
}
// upper-triangular packed index of (i <= j) in a 6x6 symmetric matrix
CEOS_HD constexpr int up21(int i, int j) { return i * 6 - (i * (i - 1)) / 2 + (j - i); }

template <typename T>
CEOS_D T tlog(T x);
template <>
CEOS_D double tlog<double>(double x) { return log(x); }
template <>
CEOS_D float tlog<float>(float x) { return logf(x); }
template <typename T>
CEOS_D T texp(T x);
template <>
CEOS_D double texp<double>(double x) { return exp(x); }
template <>
CEOS_D float texp<float>(float x) { return expf(x); }
template <typename T>
CEOS_D T tsqrt(T x);
template <>
CEOS_D double tsqrt<double>(double x) { return sqrt(x); }
template <>
CEOS_D float tsqrt<float>(float x) { return sqrtf(x); }

}  // namespace ceos
