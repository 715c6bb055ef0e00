// element_kernel.cuh -- the fused Hexa8 element loop of one Newton iteration (sm_100a).
//
// One launch replaces the reference's three serial passes over the elements:
//   SolveConstitutiveModel (FEM/Subroutines/SubSolveConstitutiveModel.f90:56-136),
//   InternalForce          (FEM/Subroutines/SubInternalForce.f90:53-85),
//   TangentStiffnessMatrix (FEM/Subroutines/SubTangentStiffnessMatrix.f90:294-311) with
//   AssembleGlobalMatrixUpperTriangular (SubAssembleGlobalMatrixUpperTriangular.f90:43-65).
//
// A CTA of 256 threads processes tiles of 32 elements:
//   gather  : thread (node n, element e) stages X, U, the CSR row starts of its node and the
//             element's slot ranks in shared memory;
//   phase A : thread (Gauss point gp, element e) forms F on the reference configuration
//             (DeformationGradient, ModElement.f90:1210-1300), the current-configuration
//             gradients (MatrixBG_ThreeDimensional, :787-889), runs the constitutive update and
//             leaves grad N, w*detJ*sigma and w*detJ*D in shared memory;
//   phase B : thread (node b, element e) accumulates over the 8 Gauss points the internal force
//             of node b (B^T sigma, ElementInternalForce :547-563) and its 3x3 stiffness blocks
//             K_ab = B_a^T D B_b + (g_a . sigma g_b) I (ElementStiffnessMatrix :320-348) for the
//             node pairs it owns, then scatters them with FP64 atomics into f_int and the upper
//             CSR through the precomputed slot map.
// Warp-uniform roles (gp or b is the warp index) keep control flow convergent; the shared
// layouts put the element index innermost so every shared access is conflict-free.
#pragma once
#include "ceos_common.cuh"
#include "materials.cuh"

namespace ceos {

constexpr int kTileE = 32;
constexpr int kThreads = 256;

// dN/dxi of the 8 nodes at the 8 Gauss points (ModElementHexa8.f90:211-268, points :278-329).
// (defined once: this header is included by a single translation unit)
__constant__ double c_dN[8][8][3];

template <typename T>
struct ElemArgs {
    int n_elem;
    const double* X;        // [3*n_nodes] reference coordinates (CoordX)
    const double* U;        // [3*n_nodes] displacements, DOF 3n+d
    const int* conn;        // [n_elem*8] 0-based node ids
    const long long* rs;    // [n_nodes] CSR position of the first entry of row 3n (0-based)
    const int* nup;         // [n_nodes] number of neighbour nodes with a larger id
    const uint32_t* ranks;  // [n_elem*8] 28 uint8 slot ranks per element (32 bytes)
    double* fint;           // [3*n_nodes]
    double* kval;           // [nnz] or nullptr (no tangent)
    const T* st_old;        // [nstate][8][n_elem]
    T* st_new;
    const T* params;        // see param_mode
    int param_mode;         // 0 uniform params[k]; 1 per element params[k*n_elem+e]; 2 per material
    int n_params;
    const int* mat_id;      // per material: params[mat_id[e]*n_params+k]
    double dt;
    uint8_t* elem_status;   // [n_elem]
    int* status_count;      // failed elements
    T* gp_stress;           // [6][8][n_elem] or nullptr
};

template <typename T>
struct __align__(16) ElemSmem {
    double x[8][3][kTileE];  // reference coordinates
    double u[8][3][kTileE];  // displacements
    long long rs[8][kTileE];
    int nup[8][kTileE];
    int node[8][kTileE];
    uint32_t ranks[kTileE][8];
    T g[8][8][3][kTileE];    // [gp][node][d][e] current-configuration gradients
    T D[8][21][kTileE];      // [gp][k][e] w*detJ*D (upper)
    T s[8][6][kTileE];       // [gp][k][e] w*detJ*sigma
    int status[kTileE];
};

template <typename T, int MODEL>
CEOS_D void run_material(const T F[3][3], const T* p, double dt, const T* st, T* stn, T sig[6], T D[21]) {
    if constexpr (MODEL == M_CNH) cnh_update<T>(F, p, sig, D);
    else if constexpr (MODEL == M_SVK) svk_update<T>(F, p, sig, D);
    else if constexpr (MODEL == M_J2_SMALL) j2_small_update<T>(F, p, st, stn, sig, D);
    else if constexpr (MODEL == M_VISCO_PRONY) visco_prony_update<T>(F, p, dt, st, stn, sig, D);
    else if constexpr (MODEL == M_J2_FINITE) j2_finite_update<T>(F, p, st, stn, sig, D);
}

template <typename T, int MODEL>
__global__ void __launch_bounds__(kThreads) element_loop_kernel(ElemArgs<T> a) {
    constexpr int NS = ModelInfo<MODEL>::nstate;
    constexpr int NP = ModelInfo<MODEL>::nparams;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ElemSmem<T>& sm = *reinterpret_cast<ElemSmem<T>*>(smem_raw);
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int n_tiles = (a.n_elem + kTileE - 1) / kTileE;

    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int e0 = tile * kTileE;
        // ---------------- gather: thread (node = warp, element = lane) ----------------------
        {
            const int e = e0 + lane;
            const int n = warp;
            if (e < a.n_elem) {
                const int node = __ldg(a.conn + (size_t)e * 8 + n);
                sm.node[n][lane] = node;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    sm.x[n][d][lane] = __ldg(a.X + 3 * (size_t)node + d);
                    sm.u[n][d][lane] = __ldg(a.U + 3 * (size_t)node + d);
                }
                sm.rs[n][lane] = __ldg(a.rs + node);
                sm.nup[n][lane] = __ldg(a.nup + node);
            }
            // slot ranks: 8 words per element, read coalesced as one 1 KB block per tile
            const int ew = t >> 3, wd = t & 7;
            if (e0 + ew < a.n_elem) sm.ranks[ew][wd] = __ldg(a.ranks + (size_t)(e0 + ew) * 8 + wd);
            if (t < kTileE) sm.status[t] = 0;
        }
        __syncthreads();

        // ---------------- phase A: thread (gp = warp, element = lane) -----------------------
        {
            const int gp = warp, el = lane, e = e0 + el;
            if (e < a.n_elem) {
                int status = 0;
                // Jacobian on the reference configuration and F = I + sum u (x) grad_X N
                T JX[3][3], Jc[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        T sx = T(0), sc = T(0);
#pragma unroll
                        for (int n = 0; n < 8; ++n) {
                            const T dn = (T)c_dN[gp][n][i];
                            const double X = sm.x[n][j][el];
                            sx += dn * (T)X;
                            sc += dn * (T)(X + sm.u[n][j][el]);
                        }
                        JX[i][j] = sx;
                        Jc[i][j] = sc;
                    }
                const T detJX = det3(JX);
                const T detJ = det3(Jc);
                if (!(detJX > T(1.0e-13)) || !(detJ > T(1.0e-13))) status |= 1;
                T JXi[3][3], Jci[3][3];
                inv3(JX, detJX, JXi);
                inv3(Jc, detJ, Jci);
                T F[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) F[i][j] = (i == j) ? T(1) : T(0);
#pragma unroll
                for (int n = 0; n < 8; ++n) {
                    const T d0 = (T)c_dN[gp][n][0], d1 = (T)c_dN[gp][n][1], d2 = (T)c_dN[gp][n][2];
                    T gX[3], gx[3];
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        gX[j] = JXi[j][0] * d0 + JXi[j][1] * d1 + JXi[j][2] * d2;
                        gx[j] = Jci[j][0] * d0 + Jci[j][1] * d1 + Jci[j][2] * d2;
                        sm.g[gp][n][j][el] = (status & 1) ? T(0) : gx[j];
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T ui = (T)sm.u[n][i][el];
#pragma unroll
                        for (int j = 0; j < 3; ++j) F[i][j] += ui * gX[j];
                    }
                }
                // constitutive update
                T p[NP];
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    if (a.param_mode == 0) p[k] = a.params[k];
                    else if (a.param_mode == 1) p[k] = a.params[(size_t)k * a.n_elem + e];
                    else p[k] = a.params[(size_t)__ldg(a.mat_id + e) * a.n_params + k];
                }
                T st[NS > 0 ? NS : 1], stn[NS > 0 ? NS : 1];
#pragma unroll
                for (int k = 0; k < NS; ++k) st[k] = a.st_old[((size_t)k * 8 + gp) * a.n_elem + e];
                T sig[6], D[21];
                if (status & 1) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) sig[k] = T(0);
#pragma unroll
                    for (int k = 0; k < 21; ++k) D[k] = T(0);
#pragma unroll
                    for (int k = 0; k < NS; ++k) stn[k] = st[k];
                } else {
                    run_material<T, MODEL>(F, p, a.dt, st, stn, sig, D);
                }
#pragma unroll
                for (int k = 0; k < NS; ++k) a.st_new[((size_t)k * 8 + gp) * a.n_elem + e] = stn[k];
                bool finite = true;
#pragma unroll
                for (int k = 0; k < 6; ++k) finite = finite && isfinite(sig[k]);
                if (!finite) status |= 4;
                if (a.gp_stress) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) a.gp_stress[((size_t)k * 8 + gp) * a.n_elem + e] = sig[k];
                }
                const T w = (status & 5) ? T(0) : detJ;  // Gauss weight is 1 (Hexa8 full integration)
#pragma unroll
                for (int k = 0; k < 6; ++k) sm.s[gp][k][el] = w * sig[k];
#pragma unroll
                for (int k = 0; k < 21; ++k) sm.D[gp][k][el] = w * D[k];
                if (status) atomicOr(&sm.status[el], status);
            }
        }
        __syncthreads();
        if (t < kTileE && e0 + t < a.n_elem) {
            const int st = sm.status[t];
            a.elem_status[e0 + t] = (uint8_t)st;
            if (st) atomicAdd(a.status_count, 1);
        }

        // ---------------- phase B: thread (node b = warp, element = lane) -------------------
        {
            const int b = warp, el = lane, e = e0 + el;
            if (e < a.n_elem) {
                const int npair = (b < 4) ? 4 : 3;  // off-diagonal partners a = b+1..b+npair (mod 8)
                T f0 = 0, f1 = 0, f2 = 0;
                T Kd[6] = {0, 0, 0, 0, 0, 0};
                T Ko[4][9];
#pragma unroll
                for (int o = 0; o < 4; ++o)
#pragma unroll
                    for (int k = 0; k < 9; ++k) Ko[o][k] = T(0);
#pragma unroll 1
                for (int gp = 0; gp < 8; ++gp) {
                    const T gx = sm.g[gp][b][0][el], gy = sm.g[gp][b][1][el], gz = sm.g[gp][b][2][el];
                    T Dm[21];
#pragma unroll
                    for (int k = 0; k < 21; ++k) Dm[k] = sm.D[gp][k][el];
                    const T s0 = sm.s[gp][0][el], s1 = sm.s[gp][1][el], s2 = sm.s[gp][2][el], s3 = sm.s[gp][3][el],
                            s4 = sm.s[gp][4][el], s5 = sm.s[gp][5][el];
                    // sigma g_b: the internal force of node b and the geometric term
                    const T q0 = s0 * gx + s3 * gy + s5 * gz;
                    const T q1 = s3 * gx + s1 * gy + s4 * gz;
                    const T q2 = s5 * gx + s4 * gy + s2 * gz;
                    f0 += q0; f1 += q1; f2 += q2;
                    // DB = D B_b (6x3), D symmetric from its upper triangle
                    T DB[6][3];
#pragma unroll
                    for (int i = 0; i < 6; ++i) {
                        const T d0 = Dm[i <= 0 ? up21(i, 0) : up21(0, i)];
                        const T d1 = Dm[i <= 1 ? up21(i, 1) : up21(1, i)];
                        const T d2 = Dm[i <= 2 ? up21(i, 2) : up21(2, i)];
                        const T d3 = Dm[i <= 3 ? up21(i, 3) : up21(3, i)];
                        const T d4 = Dm[i <= 4 ? up21(i, 4) : up21(4, i)];
                        const T d5 = Dm[i <= 5 ? up21(i, 5) : up21(5, i)];
                        DB[i][0] = d0 * gx + d3 * gy + d5 * gz;
                        DB[i][1] = d1 * gy + d3 * gx + d4 * gz;
                        DB[i][2] = d2 * gz + d4 * gy + d5 * gx;
                    }
                    // diagonal block (b,b), upper 6
                    {
                        const T geo = gx * q0 + gy * q1 + gz * q2;
                        T M[3][3];
#pragma unroll
                        for (int l = 0; l < 3; ++l) {
                            M[0][l] = gx * DB[0][l] + gy * DB[3][l] + gz * DB[5][l];
                            M[1][l] = gy * DB[1][l] + gx * DB[3][l] + gz * DB[4][l];
                            M[2][l] = gz * DB[2][l] + gy * DB[4][l] + gx * DB[5][l];
                        }
                        Kd[0] += M[0][0] + geo; Kd[1] += M[0][1]; Kd[2] += M[0][2];
                        Kd[3] += M[1][1] + geo; Kd[4] += M[1][2]; Kd[5] += M[2][2] + geo;
                    }
#pragma unroll
                    for (int o = 0; o < 4; ++o) {
                        if (o < npair) {
                            const int an = (b + 1 + o) & 7;
                            const T ax = sm.g[gp][an][0][el], ay = sm.g[gp][an][1][el], az = sm.g[gp][an][2][el];
                            const T geo = ax * q0 + ay * q1 + az * q2;
#pragma unroll
                            for (int l = 0; l < 3; ++l) {
                                Ko[o][0 * 3 + l] += ax * DB[0][l] + ay * DB[3][l] + az * DB[5][l];
                                Ko[o][1 * 3 + l] += ay * DB[1][l] + ax * DB[3][l] + az * DB[4][l];
                                Ko[o][2 * 3 + l] += az * DB[2][l] + ay * DB[4][l] + ax * DB[5][l];
                            }
                            Ko[o][0] += geo; Ko[o][4] += geo; Ko[o][8] += geo;
                        }
                    }
                }
                // ---- scatter ----
                const int Bn = sm.node[b][el];
                atomicAdd(a.fint + 3 * (size_t)Bn + 0, (double)f0);
                atomicAdd(a.fint + 3 * (size_t)Bn + 1, (double)f1);
                atomicAdd(a.fint + 3 * (size_t)Bn + 2, (double)f2);
                if (a.kval) {
                    {
                        const long long r0 = sm.rs[b][el];
                        const int m = sm.nup[b][el];
                        const long long r1 = r0 + 3 + 3 * m, r2 = r1 + 2 + 3 * m;
                        double* K = a.kval;
                        atomicAdd(K + r0 + 0, (double)Kd[0]);
                        atomicAdd(K + r0 + 1, (double)Kd[1]);
                        atomicAdd(K + r0 + 2, (double)Kd[2]);
                        atomicAdd(K + r1 + 0, (double)Kd[3]);
                        atomicAdd(K + r1 + 1, (double)Kd[4]);
                        atomicAdd(K + r2 + 0, (double)Kd[5]);
                    }
                    const uint8_t* rk = reinterpret_cast<const uint8_t*>(&sm.ranks[el][0]);
#pragma unroll
                    for (int o = 0; o < 4; ++o) {
                        if (o < npair) {
                            const int an = (b + 1 + o) & 7;
                            const int An = sm.node[an][el];
                            const int lo_local = an < b ? an : b, hi_local = an < b ? b : an;
                            const int r = rk[pair_index(lo_local, hi_local)];
                            const bool a_low = An < Bn;  // rows belong to the smaller global node
                            const int lo_n = a_low ? an : b;
                            const long long r0 = sm.rs[lo_n][el];
                            const int m = sm.nup[lo_n][el];
                            const long long row0 = r0 + 3 + 3 * r;
                            const long long row1 = r0 + (3 + 3 * m) + 2 + 3 * r;
                            const long long row2 = r0 + (3 + 3 * m) + (2 + 3 * m) + 1 + 3 * r;
                            double* K = a.kval;
                            if (a_low) {  // (3A+k, 3B+l) += M[k][l]
#pragma unroll
                                for (int l = 0; l < 3; ++l) {
                                    atomicAdd(K + row0 + l, (double)Ko[o][0 * 3 + l]);
                                    atomicAdd(K + row1 + l, (double)Ko[o][1 * 3 + l]);
                                    atomicAdd(K + row2 + l, (double)Ko[o][2 * 3 + l]);
                                }
                            } else {  // (3B+l, 3A+k) += M[k][l]
#pragma unroll
                                for (int k = 0; k < 3; ++k) {
                                    atomicAdd(K + row0 + k, (double)Ko[o][k * 3 + 0]);
                                    atomicAdd(K + row1 + k, (double)Ko[o][k * 3 + 1]);
                                    atomicAdd(K + row2 + k, (double)Ko[o][k * 3 + 2]);
                                }
                            }
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace ceos
