// fe2.cu -- batched FE^2 micro problems: many periodic RVEs solved together on one GPU.
//
// The reference solves ONE representative volume element at a time under a prescribed macro
// deformation gradient (MultiScale/ModMultiscaleAnalysis.f90:445-470, periodic constraints by
// the elimination K_red = T^T K T in FEM/Modules/ModMultiscalePeriodicFEMSoE.f90:77-182) and
// homogenizes the first Piola stress (HomogenizeStress, ModMultiscaleAnalysis.f90:140-329).  The
// batched solver here has no reference counterpart:
//   * all RVEs form one disjoint Hexa8 mesh evaluated by the fused element kernel (FP64);
//   * periodicity: node (i,j,k) of an n^3 RVE carries the fluctuation of independent node
//     (i mod n, j mod n, k mod n); independent node 0 is held fixed (rigid translation);
//     u = (Fbar - I) X + w(independent node);
//   * Newton on the fluctuations; every linear system T^T K T dw = -T^T f_int is solved by
//     fe2_minres_kernel: a persistent kernel, one CTA per RVE taken from a work queue ordered
//     by size (largest first), block-Jacobi (3x3 nodal, SPD) preconditioned MINRES in FP32
//     shared memory with FP64 iterative refinement of the residual to a relative 1e-8 (MINRES
//     rather than CG because T^T K T turns indefinite when compressed fibres buckle);
//   * Pbar = (1/V0) sum_a f_int,a (x) X_a (virtual work with the affine modes, equal to the
//     Gauss-point integral of HomogenizeStress for the same quadrature) and the 9x9 tangent
//     dPbar/dFbar = (Z^T K Z - M^T (T^T K T)^{-1} M)/V0 with M = T^T K Z (static condensation).
// Every loop has an iteration cap; no kernel waits on another CTA.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ceos_gpu.h"
#include "ceos_handle.h"

namespace {

using ceos::Handle;

constexpr int kSolveThreads = 512;
constexpr int kMaxCells = 14;  // largest RVE (cells per side) the shared-memory solver holds

struct Fe2 {
    int n_rve = 0, device = 0;
    double force_floor = 0.0;            // residual norm below which an RVE counts as converged
    int n_sub = 1;                       // macro load sub-increments per solve
    double mu_m = 1.0, mu_f = 50.0, k_over_mu = 100.0;
    int allow_failures = 0;              // 1: RVEs that cannot converge are reported, not fatal
    int solver_ctas = 0;                 // RVEs solved concurrently by the MINRES kernel (0: automatic)
    int solver_threads = kSolveThreads;  // threads per RVE of the MINRES kernel (autotuned: 256 or 512)
    // CUDA graphs of one continuation round, captured on first use and replayed every round:
    // g_assemble = Fbar upload, assembly, failed-element count, residual norms;
    // g_solve = per-RVE operations, linear solve, iteration counts, Newton step.
    // They exchange data with the host through pinned buffers at fixed addresses.
    cudaGraphExec_t g_assemble = nullptr, g_solve = nullptr;
    double* hp_Fs = nullptr;             // pinned [n_rve*9]
    double* hp_rn = nullptr;             // pinned [n_rve]
    double* hp_eta = nullptr;            // pinned [n_rve]
    int* hp_op = nullptr;                // pinned [n_rve]
    int* hp_need = nullptr;              // pinned [n_rve]
    int* hp_cgi = nullptr;               // pinned [n_rve]
    int* hp_status = nullptr;            // pinned [1] failed elements of the last assembly
    // device-resident rounds (ceos_fe2_set_device_rounds): the whole continuation is one graph, a WHILE
    // node whose body is one round (Fbar, assembly, failure flags, residual norms, the per-RVE decisions,
    // operations, linear solve, Newton step); the decision kernel keeps each RVE's continuation state on
    // the device and the last kernel of the body sets the loop condition
    int device_rounds = 1;
    cudaGraphExec_t g_rounds = nullptr;
    int* d_rs_int = nullptr;      // [8][n_rve] phase, nit, halv, cuts, its, cg_tot, spare, spare
    double* d_rs_dbl = nullptr;   // [6][n_rve] a_done, da, a_try, r0, racc, spare
    double* d_Fp = nullptr;       // [n_rve*9] start of each RVE's path
    double* d_Ft = nullptr;       // [n_rve*9] target Fbar
    int* d_rctl = nullptr;        // [4] rounds run, RVEs still in Newton this round, abort flag, RVE that aborted
    double* d_rpar = nullptr;     // [4] tol, force floor, max_newton, max_rounds (read by the round kernels)
    void drop_graphs() {
        if (g_assemble) cudaGraphExecDestroy(g_assemble);
        if (g_solve) cudaGraphExecDestroy(g_solve);
        if (g_rounds) cudaGraphExecDestroy(g_rounds);
        g_assemble = g_solve = g_rounds = nullptr;
    }
    int warm = 0;                        // 1: continue every RVE from its last converged state
    std::vector<double> F_prev;          // [n_rve][9] Fbar of the last converged state (warm start)
    std::vector<int> solve_mask;         // [n_rve] 0: RVE skipped by the next solves (empty: all solved)
    std::vector<int> n;                  // cells per side of each RVE
    std::vector<double> vf_nominal, vf_actual;
    Handle* loop = nullptr;              // element loop over the union of all RVE meshes
    int n_nodes = 0;
    long long nnz = 0;
    // per RVE offsets (host and device)
    std::vector<int> node_off, red_off, nodes_of;  // node_off[r], reduced dof offset, node count
    int n_red = 0;
    int* d_node_off = nullptr;  // [n_rve+1]
    int* d_red_off = nullptr;   // [n_rve+1]
    int* d_ncell = nullptr;     // [n_rve]
    int* d_rve_of_node = nullptr;
    int* d_rve_of_elem = nullptr;  // [n_elem]
    int* d_fail = nullptr;         // [n_rve] failed-element flag of the last assembly
    int* d_op = nullptr;           // [n_rve] per-RVE vector operation (rve_op_kernel)
    double* d_wc = nullptr;        // [n_red] fluctuations at the last converged load level
    double* d_eta = nullptr;       // [n_rve] relative tolerance of each RVE's linear solve
    int* d_fmap = nullptr;      // [3*n_nodes] global reduced dof or -1
    int* d_col = nullptr;       // [nnz] 0-based column of the upper CSR
    int* d_rcol = nullptr;      // [nnz] column as RVE-local reduced dof, -1 on the fixed node
    int* d_gcoord = nullptr;    // [n_nodes] grid coordinates of each node in its RVE (i | j<<8 | k<<16)
    int* d_rve_of_blk = nullptr;  // [n_red/3] RVE of each independent node
    float* d_kell = nullptr;    // [81 n_red] periodic ELL copy of T^T K T (FP32), slot-major per RVE
    int* d_order = nullptr;     // RVEs by decreasing size
    int* d_queue = nullptr;     // work-queue counter
    double* d_Fbar = nullptr;   // [n_rve*9] row-major
    double* d_w = nullptr;      // [n_red] fluctuations
    double* d_u = nullptr;      // [3*n_nodes]
    double* d_rhs = nullptr;    // [n_red]
    double* d_dx = nullptr;     // [n_red]
    double* d_r64 = nullptr;    // [n_red]
    double* d_y64 = nullptr;    // [3*n_nodes] FP64 SpMV scratch
    float* d_minv = nullptr;    // [n_red/3 + n_rve][9] inverse nodal diagonal blocks
    double* d_rnorm = nullptr;  // [n_rve]
    int* d_cg_iters = nullptr;  // [n_rve]
    int* d_active = nullptr;    // [n_rve]
    double* d_P = nullptr;      // [n_rve*9]
    double* d_A = nullptr;      // [n_rve*81]
    double* d_nn = nullptr;     // [n_rve] Newton residual norms
    double* d_Z = nullptr;      // [n_rve*81] Z^T K Z
    double* d_M = nullptr;      // [9*n_red] M = T^T K Z (column-major per mode)
    double* d_X9 = nullptr;     // [9*n_red] solutions of the 9 condensation systems
    std::string msg;
    ~Fe2() {
        drop_graphs();
        void* hp[] = {hp_Fs, hp_rn, hp_eta, hp_op, hp_need, hp_cgi, hp_status};
        for (void* q : hp)
            if (q) cudaFreeHost(q);
        void* p[] = {d_node_off, d_red_off, d_ncell, d_rve_of_node, d_fmap, d_col, d_order, d_queue, d_Fbar, d_w,
                     d_u, d_rhs, d_dx, d_r64, d_y64, d_minv, d_rnorm, d_cg_iters, d_active, d_P, d_A, d_nn, d_Z, d_M, d_X9,
                     d_rve_of_elem, d_fail, d_op, d_wc, d_eta, d_rcol, d_gcoord, d_rve_of_blk, d_kell,
                     d_rs_int, d_rs_dbl, d_Fp, d_Ft, d_rctl, d_rpar};
        for (void* q : p)
            if (q) cudaFree(q);
        if (loop) ceos_destroy(loop);
    }
};

#define CKF(call)                                                                  \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            f->msg = std::string(#call) + ": " + cudaGetErrorString(e_);          \
            return CEOS_E_CUDA;                                                    \
        }                                                                          \
    } while (0)

// ---------------------------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------------------------
__global__ void expand_u_kernel(int n_nodes, const double* X, const int* rve_of_node, const double* Fbar,
                                const int* fmap, const double* w, double* u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n_nodes) return;
    const int a = i / 3, d = i - 3 * a;
    const double* F = Fbar + 9 * rve_of_node[a];
    double v = (F[3 * d + 0] - (d == 0)) * X[3 * a] + (F[3 * d + 1] - (d == 1)) * X[3 * a + 1] +
               (F[3 * d + 2] - (d == 2)) * X[3 * a + 2];
    const int q = fmap[i];
    if (q >= 0) v += w[q];
    u[i] = v;
}

// T^T f: fold the full-dof vector onto the reduced dofs (sign flipped: rhs = -R)
__global__ void fold_kernel(int n_dof, const int* fmap, const double* f, double* out, double sgn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_dof) return;
    const int q = fmap[i];
    if (q >= 0) atomicAdd(out + q, sgn * f[i]);
}

// Periodic ELL copy of T^T K T: reduced row r (independent node ind = r/3 + 1, component r%3) of
// an n^3 RVE couples with the 27 periodic neighbours of its node, so its entries sit in 81 slots
// (neighbour offset nb = (di+1)*9 + (dj+1)*3 + (dk+1), column component dc): value of slot s of
// row r at kell[81 q0 + s m + r] (m reduced dofs of the RVE, q0 its first).  The fold adds every
// upper CSR entry (R, C) of the union mesh and its transpose; the offset comes from the nodes'
// unwrapped grid coordinates (nodes of one element differ by at most one cell per axis), so it is
// right for every n >= 2.
__global__ void fold_ell_kernel(int n_dof, const long long* rs, const int* nup, const int* col0, const double* K,
                                const int* fmap, const int* rve_of_node, const int* red_off, const int* gcoord,
                                float* kell) {
    const int lane = threadIdx.x & 31;
    const int R = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (R >= n_dof) return;
    const int r = fmap[R];
    if (r < 0) return;  // warp-uniform: the fixed independent node
    const int a = R / 3, k = R - 3 * a, m = nup[a];
    const long long start = rs[a] + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
    const int len = (3 - k) + 3 * m;
    const int rve = rve_of_node[a], q0 = red_off[rve], mr = red_off[rve + 1] - q0;
    float* base = kell + 81LL * q0;
    const int ga = gcoord[a];
    for (int t = lane; t < len; t += 32) {
        const int C = col0[start + t];
        const int c = fmap[C];
        if (c < 0) continue;
        const int b = C / 3, gb = gcoord[b];
        const int di = (gb & 255) - (ga & 255), dj = ((gb >> 8) & 255) - ((ga >> 8) & 255),
                  dk = (gb >> 16) - (ga >> 16);
        const int nb = (di + 1) * 9 + (dj + 1) * 3 + (dk + 1);
        const float v = (float)K[start + t];
        atomicAdd(base + (size_t)(nb * 3 + (C - 3 * b)) * mr + (r - q0), v);
        if (C != R) atomicAdd(base + (size_t)((26 - nb) * 3 + k) * mr + (c - q0), v);
    }
}

// SPD block-Jacobi preconditioner from the ELL self blocks (offset nb = 13): the inverse of each
// positive definite nodal block; a block that is not positive definite (compressed stiff fibre,
// negative geometric stiffness) falls back to the inverse of its |diagonal|, so the
// preconditioner stays symmetric positive definite.
__global__ void invert_blocks_kernel(int n_blk, const int* rve_of_blk, const int* red_off, const float* kell,
                                     float* minv) {
    const int bq = blockIdx.x * blockDim.x + threadIdx.x;
    if (bq >= n_blk) return;
    const int rve = rve_of_blk[bq], q0 = red_off[rve], m = red_off[rve + 1] - q0;
    const int r0 = 3 * bq - q0;
    const float* base = kell + 81LL * q0;
    double A[9];
    for (int dr = 0; dr < 3; ++dr)
        for (int dc = 0; dc < 3; ++dc) A[3 * dr + dc] = base[(size_t)(13 * 3 + dc) * m + r0 + dr];
    for (int i = 0; i < 3; ++i)  // symmetrise the FP32 sums
        for (int j = i + 1; j < 3; ++j) A[3 * i + j] = A[3 * j + i] = 0.5 * (A[3 * i + j] + A[3 * j + i]);
    double c[9];
    c[0] = A[4] * A[8] - A[5] * A[7];
    c[1] = A[2] * A[7] - A[1] * A[8];
    c[2] = A[1] * A[5] - A[2] * A[4];
    c[3] = A[5] * A[6] - A[3] * A[8];
    c[4] = A[0] * A[8] - A[2] * A[6];
    c[5] = A[2] * A[3] - A[0] * A[5];
    c[6] = A[3] * A[7] - A[4] * A[6];
    c[7] = A[1] * A[6] - A[0] * A[7];
    c[8] = A[0] * A[4] - A[1] * A[3];
    const double det = A[0] * c[0] + A[1] * c[3] + A[2] * c[6];
    // leading principal minors, relative to the diagonal products
    const bool pd = A[0] > 0.0 && c[8] > 1e-6 * A[0] * A[4] && det > 1e-6 * A[0] * A[4] * A[8];
    float* M = minv + 9 * (size_t)bq;
    if (pd) {
        const double r = 1.0 / det;
        for (int q = 0; q < 9; ++q) M[q] = (float)(c[q] * r);
    } else {
        const double amax = fmax(fabs(A[0]), fmax(fabs(A[4]), fabs(A[8])));
        const double fl = amax > 0.0 ? 1e-6 * amax : 1.0;
        for (int q = 0; q < 9; ++q) M[q] = 0.f;
        M[0] = (float)(1.0 / fmax(fabs(A[0]), fl));
        M[4] = (float)(1.0 / fmax(fabs(A[4]), fl));
        M[8] = (float)(1.0 / fmax(fabs(A[8]), fl));
    }
}

// per-RVE Euclidean norm of a reduced vector (one CTA per RVE)
__device__ __forceinline__ double block_sum_d(double v, double* red);
__global__ void rve_norm_kernel(int n_rve, const int* red_off, const double* v, double* out) {
    __shared__ double red[32];
    const int rve = blockIdx.x;
    double s = 0.0;
    for (int q = red_off[rve] + threadIdx.x; q < red_off[rve + 1]; q += blockDim.x) s += v[q] * v[q];
    s = block_sum_d(s, red);
    if (threadIdx.x == 0) out[rve] = sqrt(s);
}

// RVEs with a failed element (det J <= 1e-13) in the last element-loop evaluation
__global__ void rve_fail_kernel(int n_elem, const uint8_t* elem_status, const int* rve_of_elem, int* fail) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n_elem && elem_status[e]) atomicOr(fail + rve_of_elem[e], 1);
}
// Per-RVE operations on the reduced vectors (one CTA per RVE):
//   1 backtrack: w -= dx/2, dx /= 2   2 restore: w = wc   3 save: wc = w
enum { kOpNone = 0, kOpBacktrack = 1, kOpRestore = 2, kOpSave = 3 };
__global__ void rve_op_kernel(int n_rve, const int* red_off, const int* op, double* w, double* dx, double* wc) {
    const int rve = blockIdx.x;
    const int o = op[rve];
    if (o == kOpNone) return;
    for (int q = red_off[rve] + threadIdx.x; q < red_off[rve + 1]; q += blockDim.x) {
        if (o == kOpBacktrack) {
            w[q] -= 0.5 * dx[q];
            dx[q] *= 0.5;
        } else if (o == kOpRestore) {
            w[q] = wc[q];
        } else {
            wc[q] = w[q];
        }
    }
}

// Load continuation of every RVE (the host-driven and the device-resident rounds use the same rules):
// a Newton step is accepted when no element folds and the residual grows by at most kGrowth (never
// beyond kDiverge x the residual at the start of the load step), otherwise halved up to kMaxHalvings
// times; a load step that still fails, or does not converge in max_newton iterations, is cut back by
// the golden ratio, at most kMaxCutbacks times.
constexpr int kMaxHalvings = 6, kMaxCutbacks = 16;
constexpr double kGrowth = 1.5, kDiverge = 1e3, kGolden = 0.6180339887498949;
enum { kNewton = 0, kDone = 1, kFailed = 2 };

// One RVE's continuation state and the decision of one round on it, shared by the host-driven and the
// device-resident rounds.  rn: the RVE's residual norm after this round's assembly; ok: no element folded
// and rn is finite.  Sets op (vector operation), need (a linear solve follows) and eta (its forcing
// term); returns the flags kRejected (a halving), kCut (a load cut-back) and kExhausted (the cut-back
// limit was passed: the RVE returns to its converged state and counts as failed).
struct RveCont {
    int phase, nit, halv, cuts, its;
    double a_done, da, a_try, r0, racc;
};
enum { kRejected = 1, kCut = 2, kExhausted = 4 };
__host__ __device__ inline int decide_rve(RveCont& c, double rn, bool ok, double tol, double floor_, int max_newton,
                                          int& op, int& need, double& eta) {
    op = kOpNone;
    need = 0;
    bool cut = false, accepted = false;
    if (c.nit == 0) {  // start of a load step from the converged fluctuations
        if (!ok) cut = true;
        else { c.r0 = rn > 1e-300 ? rn : 1e-300; accepted = true; }
    } else if (ok && rn <= kGrowth * c.racc && rn <= kDiverge * c.r0) {
        accepted = true;
    } else if (c.halv >= kMaxHalvings) {
        cut = true;
    } else {
        op = kOpBacktrack;
        ++c.halv;
        return kRejected;
    }
    if (accepted) {
        c.racc = rn;
        c.halv = 0;
        if (rn <= tol * c.r0 || rn <= floor_) {
            c.a_done = c.a_try;
            op = kOpSave;
            c.nit = 0;
            if (c.a_done >= 1.0) {
                c.phase = kDone;
            } else {
                c.da = fmin(2.0 * c.da, 1.0 - c.a_done);  // grow after a converged step
                c.a_try = 1.0 - (c.a_done + c.da) < 1e-12 ? 1.0 : c.a_done + c.da;
            }
        } else if (c.nit >= max_newton) {
            cut = true;
        } else {
            // Eisenstat-Walker forcing: quadratic convergence without over-solving
            const double rel = rn / c.r0;
            eta = fmin(1e-2, fmax(rel, 0.1 * tol / rel));
            need = 1;
            ++c.nit;
            ++c.its;
        }
    }
    if (!cut) return 0;
    op = kOpRestore;
    if (++c.cuts > kMaxCutbacks) {  // give up on this RVE: back to its last converged state
        c.phase = kFailed;
        c.a_try = c.a_done;
        return kExhausted;
    }
    c.da *= kGolden;
    c.a_try = c.a_done + c.da;
    c.nit = 0;
    c.halv = 0;
    return kCut;
}

// ---- device-resident rounds ----
// state: si = [phase, nit, halv, cuts, its, cg_tot] x n_rve (ints), sd = [a_done, da, a_try, r0, racc] x
// n_rve (doubles); par = {tol, force floor, max_newton, max_rounds}; ctl = {rounds run, RVEs in Newton
// this round, abort, RVE that aborted}.

// Fbar of this round's trial load level; clears the failed-element flags.
__global__ void round_fbar_kernel(int n_rve, const double* Fp, const double* Ft, const double* sd, double* Fbar,
                                  int* fail) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * n_rve) return;
    const int r = i / 9;
    const double a = sd[2 * n_rve + r];
    Fbar[i] = Fp[i] + a * (Ft[i] - Fp[i]);
    if (i % 9 == 0) fail[r] = 0;
}

// Failed-element flags per RVE, only when the assembly reported failed elements.
__global__ void round_fail_kernel(int n_elem, const int* status_count, const uint8_t* elem_status,
                                  const int* rve_of_elem, int* fail) {
    if (*status_count == 0) return;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n_elem && elem_status[e]) atomicOr(fail + rve_of_elem[e], 1);
}

// The per-RVE decision of one round (decide_rve, one thread per RVE): operation, whether a linear
// solve is needed, and its forcing term.
__global__ void round_decide_kernel(int n_rve, int allow_failures, const double* par, const double* rn_all,
                                    const int* fail, int* si, double* sd, int* op, int* need, double* eta, int* ctl) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rve) return;
    op[r] = kOpNone;
    need[r] = 0;
    if (si[r] != kNewton) return;
    atomicAdd(ctl + 1, 1);
    RveCont c{si[r], si[n_rve + r], si[2 * n_rve + r], si[3 * n_rve + r], si[4 * n_rve + r],
              sd[r], sd[n_rve + r], sd[2 * n_rve + r], sd[3 * n_rve + r], sd[4 * n_rve + r]};
    const double rn = rn_all[r];
    int o = kOpNone, nd = 0;
    double e = eta[r];
    const int flags = decide_rve(c, rn, !fail[r] && isfinite(rn), par[0], par[1], (int)par[2], o, nd, e);
    if ((flags & kExhausted) && !allow_failures) {
        atomicCAS(ctl + 3, -1, r);
        ctl[2] = 1;
    }
    op[r] = o;
    need[r] = nd;
    eta[r] = e;
    si[r] = c.phase;
    si[n_rve + r] = c.nit;
    si[2 * n_rve + r] = c.halv;
    si[3 * n_rve + r] = c.cuts;
    si[4 * n_rve + r] = c.its;
    sd[r] = c.a_done;
    sd[n_rve + r] = c.da;
    sd[2 * n_rve + r] = c.a_try;
    sd[3 * n_rve + r] = c.r0;
    sd[4 * n_rve + r] = c.racc;
}

// End of a round: MINRES iterations of the solved RVEs, the round count, and the loop condition (another
// round while some RVE was still in Newton, no abort, and the round cap is not reached).
__global__ void round_finish_kernel(int n_rve, const int* need, const int* cg_iters, int* si, const double* par,
                                    int* ctl, cudaGraphConditionalHandle cond) {
    int* cg_tot = si + 5 * n_rve;
    for (int r = threadIdx.x; r < n_rve; r += blockDim.x)
        if (need[r]) cg_tot[r] += cg_iters[r];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int rounds = ++ctl[0];
        const bool more = ctl[1] > 0 && ctl[2] == 0 && rounds < (int)par[3];
        ctl[1] = 0;
        cudaGraphSetConditional(cond, more ? 1u : 0u);
    }
}

// w += dx on the RVEs that solved for a Newton correction
__global__ void rve_step_kernel(int n_rve, const int* red_off, const int* sel, const double* dx, double* w) {
    const int rve = blockIdx.x;
    if (!sel[rve]) return;
    for (int q = red_off[rve] + threadIdx.x; q < red_off[rve + 1]; q += blockDim.x) w[q] += dx[q];
}

// ---------------------------------------------------------------------------------------------
// persistent block-Jacobi MINRES: one CTA per RVE
// ---------------------------------------------------------------------------------------------
// T^T K T is symmetric but INDEFINITE once the stiff fibres are compressed past their
// micro-buckling load (negative geometric stiffness), where CG breaks down.  MINRES (Paige and
// Saunders, SIAM J. Numer. Anal. 12, 1975) minimises the residual over the same Krylov space at
// the same cost per iteration (one SpMV, two block reductions) and only needs a symmetric
// positive definite preconditioner.
struct SolveArgs {
    int n_rve, max_inner, max_outer;
    double inner_floor;    // smallest relative reduction asked of one FP32 cycle
    const double* eta;     // [n_rve] target relative residual of each RVE's solve
    const int* order;      // RVE indices, largest first
    int* queue;            // work counter
    const int* active;     // RVE participates in this solve
    const int* node_off;   // [n_rve+1]
    const int* red_off;    // [n_rve+1]
    const int* fmap;       // full dof -> global reduced dof or -1
    const long long* rs;   // CSR row start of row 3a
    const int* nup;
    const int* rcol;       // [nnz] column mapped to the RVE-local reduced dof, or -1
    const double* K;       // upper CSR values (FP64), refinement residuals
    const float* kell;     // periodic ELL copy in FP32, inner iterations
    const int* ncell;      // [n_rve] cells per side
    const float* minv;     // SPD block-Jacobi inverse per independent node
    int nrhs;              // right-hand sides solved one after another
    const double* rhs;     // [nrhs][n_red]
    double* x;             // [nrhs][n_red] solution
    double* r64;           // [n_red] FP64 residual scratch
    int* iters;            // [n_rve] total inner iterations (last rhs)
    double* rnorm;         // [n_rve] final relative residual (last rhs)
    int n_red;
};

__device__ __forceinline__ float block_sum_f(float v, float* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    float s = 0.f;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) red[0] = s;
    }
    __syncthreads();
    return red[0];
}
__device__ __forceinline__ double block_sum_d(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) red[0] = s;
    }
    __syncthreads();
    return red[0];
}

// y += T^T K T x over the full rows of one RVE, directly in its local reduced numbering (warp
// per full row, lanes over the row's upper entries, the transposed half by shared atomics).
// Two different dofs of one element never map to the same reduced dof for n >= 2 (periodic
// images are n cells apart), so c == ir only on the diagonal.
template <typename V, typename KV>
__device__ void rve_spmv_red(int row0, int nrow, int q0, const int* fmap, const long long* rs, const int* nup,
                             const int* rcol, const KV* K, const V* x, V* y) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int lr = warp; lr < nrow; lr += nw) {
        const int row = row0 + lr;
        const int g = fmap[row];
        if (g < 0) continue;  // the fixed independent node (warp-uniform)
        const int ir = g - q0;
        const int a = row / 3, k = row - 3 * a;
        const int m = nup[a];
        const long long start = rs[a] + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
        const int len = (3 - k) + 3 * m;
        const V xr = x[ir];
        V acc = 0;
        for (int p = lane; p < len; p += 32) {
            const int c = rcol[start + p];
            if (c < 0) continue;
            const V v = (V)K[start + p];
            acc += v * x[c];
            if (c != ir) atomicAdd(y + c, v * xr);
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(y + ir, acc);
    }
}

// y = T^T K T x over one RVE from its periodic ELL copy: thread per reduced row, the 27 neighbour
// nodes from the row's grid position (no index arrays, no atomics), slot-major coalesced values.
__device__ __forceinline__ void ell_spmv(int m, int n, const float* __restrict__ kell, const float* x, float* y) {
    const int nn = n * n;
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const int ind = r / 3 + 1;
        const int i0 = ind % n, j0 = (ind / n) % n, k0 = ind / nn;
        float acc = 0.f;
#pragma unroll
        for (int nb = 0; nb < 27; ++nb) {
            int ii = i0 + nb / 9 - 1, jj = j0 + (nb / 3) % 3 - 1, kk = k0 + nb % 3 - 1;
            ii += ii < 0 ? n : (ii >= n ? -n : 0);
            jj += jj < 0 ? n : (jj >= n ? -n : 0);
            kk += kk < 0 ? n : (kk >= n ? -n : 0);
            const int ind2 = kk * nn + jj * n + ii;
            // the fixed independent node (ind2 = 0) contributes nothing; branch-free, so that the
            // 81 independent loads of the row stay in flight together
            const float on = ind2 ? 1.f : 0.f;
            const int b = ind2 ? 3 * (ind2 - 1) : 0;
            acc += on * (__ldg(kell + (size_t)(nb * 3) * m + r) * x[b] + __ldg(kell + (size_t)(nb * 3 + 1) * m + r) * x[b + 1] +
                         __ldg(kell + (size_t)(nb * 3 + 2) * m + r) * x[b + 2]);
        }
        y[r] = acc;
    }
}

__device__ __forceinline__ void apply_block(const float* Mb, const float r[3], float z[3]) {
    z[0] = Mb[0] * r[0] + Mb[1] * r[1] + Mb[2] * r[2];
    z[1] = Mb[3] * r[0] + Mb[4] * r[1] + Mb[5] * r[2];
    z[2] = Mb[6] * r[0] + Mb[7] * r[1] + Mb[8] * r[2];
}

__global__ void __launch_bounds__(kSolveThreads) fe2_minres_kernel(SolveArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red_d[32];
    __shared__ float red_f[32];
    __shared__ int rve_s;
    const int tid = threadIdx.x, bs = blockDim.x;
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(A.queue, 1);
            rve_s = t < A.n_rve ? A.order[t] : -1;
        }
        __syncthreads();
        const int rve = rve_s;
        __syncthreads();
        if (rve < 0) return;
        const int na0 = A.node_off[rve], na1 = A.node_off[rve + 1];
        const int nf = 3 * (na1 - na0), dof0 = 3 * na0;
        const int q0 = A.red_off[rve], m = A.red_off[rve + 1] - q0, nb3 = m / 3;
        if (!A.active[rve]) continue;  // x of RVEs not solving is left as it is
        const float* Mr = A.minv + 3 * (size_t)q0;  // block of independent node j at Mr + 9 j
        const float* kell = A.kell + 81LL * q0;
        const int ncell = A.ncell[rve];
        // shared views: FP32 inner phase [xs][bufA][bufB][bufC][v][wa][wb] (m each);
        // FP64 refinement phase [xd][yd] (m each) over the same bytes
        float* xs = reinterpret_cast<float*>(smem);
        float* bufA = xs + m;
        float* bufB = bufA + m;
        float* bufC = bufB + m;
        float* v = bufC + m;
        float* wa = v + m;
        float* wb = wa + m;
        double* xd = reinterpret_cast<double*>(smem);
        double* yd = xd + m;
        for (int rh = 0; rh < A.nrhs; ++rh) {
            const double* b = A.rhs + (size_t)rh * A.n_red + q0;
            double* x = A.x + (size_t)rh * A.n_red + q0;
            double* r64 = A.r64 + q0;
            double bb = 0.0;
            for (int i = tid; i < m; i += bs) { x[i] = 0.0; r64[i] = b[i]; bb += b[i] * b[i]; }
            const double nb = sqrt(block_sum_d(bb, red_d));
            int total_it = 0;
            double rel = nb > 0.0 ? 1.0 : 0.0;
            const double eta = A.eta[rve];
            for (int outer = 0; outer < A.max_outer && nb > 0.0 && rel > eta; ++outer) {
                // ---- inner FP32 MINRES on the current FP64 residual scaled to unit norm ----
                double rr = 0.0;
                for (int i = tid; i < m; i += bs) rr += r64[i] * r64[i];
                const double nr = sqrt(block_sum_d(rr, red_d));
                const double sc = 1.0 / nr;
                // this cycle aims a little below the target, but no lower than FP32 can reach
                const float cyc_tol = (float)fmax(0.5 * eta * nb / nr, A.inner_floor);
                float* r1 = bufA;
                float* r2 = bufB;
                float* y = bufC;
                float b1 = 0.f;
                for (int j = tid; j < nb3; j += bs) {
                    float rv[3], z[3];
                    for (int c = 0; c < 3; ++c) rv[c] = (float)(r64[3 * j + c] * sc);
                    apply_block(Mr + 9 * (size_t)j, rv, z);
                    for (int c = 0; c < 3; ++c) {
                        r1[3 * j + c] = rv[c];
                        r2[3 * j + c] = rv[c];
                        y[3 * j + c] = z[c];
                        xs[3 * j + c] = 0.f;
                        wa[3 * j + c] = 0.f;
                        wb[3 * j + c] = 0.f;
                    }
                    b1 += rv[0] * z[0] + rv[1] * z[1] + rv[2] * z[2];
                }
                b1 = block_sum_f(b1, red_f);
                const float beta1 = b1 > 0.f ? sqrtf(b1) : 0.f;
                float beta = beta1, oldb = 0.f, dbar = 0.f, epsln = 0.f, phibar = beta1, cs = -1.f, sn = 0.f;
                int it = 0;
                while (it < A.max_inner && beta > 0.f) {
                    // v = y / beta;  y = K_red v - (beta/oldb) r1
                    const float s = 1.f / beta;
                    for (int i = tid; i < m; i += bs) v[i] = s * y[i];
                    __syncthreads();
                    ell_spmv(m, ncell, kell, v, y);
                    __syncthreads();
                    const float f1 = it > 0 ? beta / oldb : 0.f;
                    float al = 0.f;
                    for (int i = tid; i < m; i += bs) {
                        const float yi = y[i] - f1 * r1[i];
                        y[i] = yi;
                        al += v[i] * yi;
                    }
                    const float alfa = block_sum_f(al, red_f);
                    // y -= (alfa/beta) r2;  z = M y into r1's buffer;  beta = sqrt(y . z)
                    const float f2 = alfa / beta;
                    float bt = 0.f;
                    for (int j = tid; j < nb3; j += bs) {
                        float yv[3], z[3];
                        for (int c = 0; c < 3; ++c) {
                            yv[c] = y[3 * j + c] - f2 * r2[3 * j + c];
                            y[3 * j + c] = yv[c];
                        }
                        apply_block(Mr + 9 * (size_t)j, yv, z);
                        for (int c = 0; c < 3; ++c) r1[3 * j + c] = z[c];
                        bt += yv[0] * z[0] + yv[1] * z[1] + yv[2] * z[2];
                    }
                    bt = block_sum_f(bt, red_f);
                    {  // rotate: r1 <- r2, r2 <- y, y <- z
                        float* t = r1;
                        r1 = r2;
                        r2 = y;
                        y = t;
                    }
                    oldb = beta;
                    beta = bt > 0.f ? sqrtf(bt) : 0.f;
                    // Givens rotation of the tridiagonal Lanczos matrix
                    const float oldeps = epsln;
                    const float delta = cs * dbar + sn * alfa;
                    const float gbar = sn * dbar - cs * alfa;
                    epsln = sn * beta;
                    dbar = -cs * beta;
                    const float gamma = fmaxf(sqrtf(gbar * gbar + beta * beta), 1e-30f);
                    cs = gbar / gamma;
                    sn = beta / gamma;
                    const float phi = cs * phibar;
                    phibar *= sn;
                    const float dn = 1.f / gamma;
                    for (int i = tid; i < m; i += bs) {
                        const float t = wa[i];
                        const float wn = (v[i] - oldeps * wb[i] - delta * t) * dn;
                        wb[i] = t;
                        wa[i] = wn;
                        xs[i] += phi * wn;
                    }
                    ++it;
                    if (phibar < cyc_tol * beta1) break;
                }
                total_it += it;
                // ---- FP64 refinement: x += nr * xs; r64 = b - K_red x ----
                __syncthreads();
                for (int i = tid; i < m; i += bs) x[i] += nr * (double)xs[i];
                __syncthreads();
                for (int i = tid; i < m; i += bs) { xd[i] = x[i]; yd[i] = 0.0; }
                __syncthreads();
                rve_spmv_red<double, double>(dof0, nf, q0, A.fmap, A.rs, A.nup, A.rcol, A.K, xd, yd);
                __syncthreads();
                double rs2 = 0.0;
                for (int i = tid; i < m; i += bs) {
                    const double ri = b[i] - yd[i];
                    r64[i] = ri;
                    rs2 += ri * ri;
                }
                rel = sqrt(block_sum_d(rs2, red_d)) / nb;
            }
            if (tid == 0) {
                A.iters[rve] = total_it;
                A.rnorm[rve] = rel;
            }
            __syncthreads();
        }
    }
}

// Homogenized first Piola stress and the Z^T K Z term, one CTA per RVE.
//   Pbar_iJ = (1/V0) sum_a f_{a,i} X_{a,J};  (Z^T K Z)_{iJ,kL} = sum_a X_{a,J} (K z_kL)_{a,i}
__global__ void homogenize_kernel(int n_rve, const int* node_off, const double* X, const double* f, double* P,
                                  double V0) {
    __shared__ double red[32];
    const int rve = blockIdx.x;
    if (rve >= n_rve) return;
    const int a0 = node_off[rve], a1 = node_off[rve + 1];
    for (int c = 0; c < 9; ++c) {
        const int i = c / 3, J = c % 3;
        double s = 0.0;
        for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) s += f[3 * a + i] * X[3 * a + J];
        s = block_sum_d(s, red);
        if (threadIdx.x == 0) P[9 * rve + c] = s / V0;
    }
}

// Affine mode z_kL (u_{a,k} = X_{a,L}) of every RVE into u; y = K_sym u computed by a plain
// upper-CSR SpMV with FP64 atomics.
__global__ void affine_mode_kernel(int n_nodes, const double* X, int kL, double* u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n_nodes) return;
    const int a = i / 3, d = i - 3 * a, k = kL / 3, L = kL % 3;
    u[i] = d == k ? X[3 * a + L] : 0.0;
}
__global__ void spmv_upper_kernel(int n_dof, const long long* rs, const int* nup, const int* col, const double* K,
                                  const double* x, double* y) {
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= n_dof) return;
    const int a = row / 3, k = row - 3 * a;
    const int m = nup[a];
    const long long start = rs[a] + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
    const int len = (3 - k) + 3 * m;
    const double xr = x[row];
    double acc = 0.0;
    for (int p = lane; p < len; p += 32) {
        const int c = col[start + p];
        const double v = K[start + p];
        acc += v * x[c];
        if (c != row) atomicAdd(y + c, v * xr);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) atomicAdd(y + row, acc);
}
// ZKZ_{iJ,kL} += sum_a X_{a,J} y_{a,i}
__global__ void zkz_kernel(int n_rve, const int* node_off, const double* X, const double* y, int kL, double* Z,
                           double V0) {
    __shared__ double red[32];
    const int rve = blockIdx.x;
    const int a0 = node_off[rve], a1 = node_off[rve + 1];
    for (int c = 0; c < 9; ++c) {
        const int i = c / 3, J = c % 3;
        double s = 0.0;
        for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) s += y[3 * a + i] * X[3 * a + J];
        s = block_sum_d(s, red);
        if (threadIdx.x == 0) Z[81 * rve + 9 * c + kL] = s / V0;
    }
}
// A_{iJ,kL} = ZKZ - (1/V0) sum_q M_iJ[q] X_kL[q] per RVE
__global__ void condense_kernel(int n_rve, const int* red_off, int n_red, const double* M, const double* Xs,
                                const double* Z, double* A, double V0) {
    __shared__ double red[32];
    const int rve = blockIdx.x;
    const int q0 = red_off[rve], q1 = red_off[rve + 1];
    for (int c = 0; c < 81; ++c) {
        const int u = c / 9, v = c % 9;
        double s = 0.0;
        for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) s += M[(size_t)u * n_red + q] * Xs[(size_t)v * n_red + q];
        s = block_sum_d(s, red);
        if (threadIdx.x == 0) A[81 * rve + c] = Z[81 * rve + c] - s / V0;
    }
}

// shared memory of the solver: 7 FP32 vectors (or 2 FP64 vectors) of the largest reduced size
size_t solve_smem_bytes(int max_m) { return std::max(sizeof(float) * 7, sizeof(double) * 2) * (size_t)max_m; }

// Solve T^T K T x = rhs for the RVEs flagged in d_active, each to its relative tolerance d_eta.
int run_solver(Fe2* f, int nrhs, const double* rhs, double* x, int max_inner, int max_outer) {
    Handle* h = f->loop;
    int max_m = 0;
    for (int r = 0; r < f->n_rve; ++r) max_m = std::max(max_m, f->red_off[r + 1] - f->red_off[r]);
    const size_t smem = solve_smem_bytes(max_m);
    CKF(cudaFuncSetAttribute(fe2_minres_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device);
    const int bs = f->solver_threads;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fe2_minres_kernel, bs, smem);
    SolveArgs a;
    a.n_rve = f->n_rve;
    a.max_inner = max_inner;
    a.max_outer = max_outer;
    a.inner_floor = 1e-4;
    a.eta = f->d_eta;
    a.order = f->d_order;
    a.queue = f->d_queue;
    a.active = f->d_active;
    a.node_off = f->d_node_off;
    a.red_off = f->d_red_off;
    a.fmap = f->d_fmap;
    a.rs = h->d_rs;
    a.nup = h->d_nup;
    a.rcol = f->d_rcol;
    a.K = h->d_kval;
    a.kell = f->d_kell;
    a.ncell = f->d_ncell;
    a.minv = f->d_minv;
    a.nrhs = nrhs;
    a.rhs = rhs;
    a.x = x;
    a.r64 = f->d_r64;
    a.iters = f->d_cg_iters;
    a.rnorm = f->d_rnorm;
    a.n_red = f->n_red;
    CKF(cudaMemsetAsync(f->d_queue, 0, sizeof(int), h->stream));
    // RVEs in flight: as many as occupancy allows (bounding them to keep the ELL copies within L2,
    // one per SM, measured slower: 2.33 s vs 1.54 s for 512 RVEs of n = 8), or the caller's number
    int grid = std::max(1, std::min(f->n_rve, sms * std::max(per_sm, 1)));
    if (f->solver_ctas > 0) grid = std::max(1, std::min(grid, f->solver_ctas));
    fe2_minres_kernel<<<grid, bs, smem, h->stream>>>(a);
    CKF(cudaGetLastError());
    return 0;
}

// Newton iteration pieces: u, element loop (f_int, K), rhs = -T^T f_int, block-Jacobi inverse.
int assemble(Fe2* f) {
    Handle* h = f->loop;
    const int nd = 3 * f->n_nodes;
    expand_u_kernel<<<(nd + 255) / 256, 256, 0, h->stream>>>(f->n_nodes, h->d_X, f->d_rve_of_node, f->d_Fbar,
                                                              f->d_fmap, f->d_w, f->d_u);
    CKF(cudaGetLastError());
    int rc = ceos::evaluate_device(h, 0.0, f->d_u, h->d_fint, h->d_kval, h->stream);
    if (rc) return rc;
    CKF(cudaMemsetAsync(f->d_rhs, 0, sizeof(double) * f->n_red, h->stream));
    fold_kernel<<<(nd + 255) / 256, 256, 0, h->stream>>>(nd, f->d_fmap, h->d_fint, f->d_rhs, -1.0);
    CKF(cudaGetLastError());
    const int n_blk = f->n_red / 3;
    CKF(cudaMemsetAsync(f->d_kell, 0, sizeof(float) * 81 * (size_t)f->n_red, h->stream));
    fold_ell_kernel<<<(unsigned)(((long long)nd * 32 + 255) / 256), 256, 0, h->stream>>>(
        nd, h->d_rs, h->d_nup, f->d_col, h->d_kval, f->d_fmap, f->d_rve_of_node, f->d_red_off, f->d_gcoord, f->d_kell);
    CKF(cudaGetLastError());
    invert_blocks_kernel<<<(n_blk + 255) / 256, 256, 0, h->stream>>>(n_blk, f->d_rve_of_blk, f->d_red_off, f->d_kell,
                                                                      f->d_minv);
    CKF(cudaGetLastError());
    return 0;
}

// The device work of one continuation round, recorded once into CUDA graphs (stream capture) and
// replayed every round; the host exchanges Fbar, operations, tolerances, norms and iteration counts
// through the pinned hp_* buffers.
int record_assemble(Fe2* f) {
    Handle* h = f->loop;
    cudaStream_t s = h->stream;
    const int nr = f->n_rve;
    CKF(cudaMemcpyAsync(f->d_Fbar, f->hp_Fs, sizeof(double) * 9 * nr, cudaMemcpyHostToDevice, s));
    const int rc = assemble(f);
    if (rc) return rc;
    CKF(cudaMemcpyAsync(f->hp_status, h->d_status_count, sizeof(int), cudaMemcpyDeviceToHost, s));
    rve_norm_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_rhs, f->d_nn);
    CKF(cudaGetLastError());
    CKF(cudaMemcpyAsync(f->hp_rn, f->d_nn, sizeof(double) * nr, cudaMemcpyDeviceToHost, s));
    return 0;
}

int record_solve(Fe2* f) {
    Handle* h = f->loop;
    cudaStream_t s = h->stream;
    const int nr = f->n_rve;
    CKF(cudaMemcpyAsync(f->d_op, f->hp_op, sizeof(int) * nr, cudaMemcpyHostToDevice, s));
    rve_op_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_op, f->d_w, f->d_dx, f->d_wc);
    CKF(cudaGetLastError());
    CKF(cudaMemcpyAsync(f->d_active, f->hp_need, sizeof(int) * nr, cudaMemcpyHostToDevice, s));
    CKF(cudaMemcpyAsync(f->d_eta, f->hp_eta, sizeof(double) * nr, cudaMemcpyHostToDevice, s));
    const int rc = run_solver(f, 1, f->d_rhs, f->d_dx, 2000, 3);  // an inexact step is still a descent try
    if (rc) return rc;
    CKF(cudaMemcpyAsync(f->hp_cgi, f->d_cg_iters, sizeof(int) * nr, cudaMemcpyDeviceToHost, s));
    rve_step_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_active, f->d_dx, f->d_w);
    CKF(cudaGetLastError());
    return 0;
}

// Capture record(f) on the handle's stream into *exec (nothing is executed while capturing).
int capture(Fe2* f, int (*record)(Fe2*), cudaGraphExec_t* exec) {
    cudaStream_t s = f->loop->stream;
    CKF(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    const int rc = record(f);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);  // always ends the capture, also after an error
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        f->msg = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
        return CEOS_E_CUDA;
    }
    const cudaError_t e2 = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
        *exec = nullptr;
        f->msg = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2);
        return CEOS_E_CUDA;
    }
    return 0;
}

// One device-resident round, recorded into the body of the WHILE node (no host buffers: everything
// the round needs lives on the device).
int record_round(Fe2* f, cudaGraphConditionalHandle cond) {
    Handle* h = f->loop;
    cudaStream_t s = h->stream;
    const int nr = f->n_rve;
    round_fbar_kernel<<<(9 * nr + 255) / 256, 256, 0, s>>>(nr, f->d_Fp, f->d_Ft, f->d_rs_dbl, f->d_Fbar, f->d_fail);
    CKF(cudaGetLastError());
    int rc = assemble(f);
    if (rc) return rc;
    round_fail_kernel<<<(h->n_elem + 255) / 256, 256, 0, s>>>(h->n_elem, h->d_status_count, h->d_elem_status,
                                                              f->d_rve_of_elem, f->d_fail);
    rve_norm_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_rhs, f->d_nn);
    round_decide_kernel<<<(nr + 255) / 256, 256, 0, s>>>(nr, f->allow_failures, f->d_rpar, f->d_nn, f->d_fail,
                                                         f->d_rs_int, f->d_rs_dbl, f->d_op, f->d_active, f->d_eta,
                                                         f->d_rctl);
    rve_op_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_op, f->d_w, f->d_dx, f->d_wc);
    CKF(cudaGetLastError());
    rc = run_solver(f, 1, f->d_rhs, f->d_dx, 2000, 3);  // RVEs without need[] skip the solve
    if (rc) return rc;
    rve_step_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_active, f->d_dx, f->d_w);
    round_finish_kernel<<<1, 256, 0, s>>>(nr, f->d_active, f->d_cg_iters, f->d_rs_int, f->d_rpar, f->d_rctl, cond);
    CKF(cudaGetLastError());
    return 0;
}

// The whole continuation as one graph: a WHILE node (condition 1 at every launch) around one round.
int build_round_graph(Fe2* f) {
    cudaStream_t s = f->loop->stream;
    const int nr = f->n_rve;
    if (!f->d_rs_int) {
        CKF(cudaMalloc(&f->d_rs_int, sizeof(int) * 8 * (size_t)nr));
        CKF(cudaMalloc(&f->d_rs_dbl, sizeof(double) * 6 * (size_t)nr));
        CKF(cudaMalloc(&f->d_Fp, sizeof(double) * 9 * (size_t)nr));
        CKF(cudaMalloc(&f->d_Ft, sizeof(double) * 9 * (size_t)nr));
        CKF(cudaMalloc(&f->d_rctl, sizeof(int) * 4));
        CKF(cudaMalloc(&f->d_rpar, sizeof(double) * 4));
    }
    cudaGraph_t g = nullptr;
    CKF(cudaGraphCreate(&g, 0));
    auto fail = [&](const char* what, cudaError_t e) {
        f->msg = std::string(what) + ": " + cudaGetErrorString(e);
        cudaGraphDestroy(g);
        return CEOS_E_CUDA;
    };
    cudaGraphConditionalHandle cond;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return fail("cudaGraphConditionalHandleCreate", e);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    if (e != cudaSuccess) return fail("cudaGraphAddNode (while)", e);
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return fail("cudaStreamBeginCaptureToGraph", e);
    const int rc = record_round(f, cond);
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(s, &out);  // always ends the capture, also after an error
    if (rc) {
        cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail("cudaStreamEndCapture", e);
    e = cudaGraphInstantiate(&f->g_rounds, g, 0);
    if (e != cudaSuccess) {
        f->g_rounds = nullptr;
        return fail("cudaGraphInstantiate (rounds)", e);
    }
    cudaGraphDestroy(g);
    return 0;
}

// Fibre area fraction of cell column (i, j) of an n^3 RVE: share of 16 x 16 sub-points of the
// cell's cross-section strictly inside the fibre circle x^2 + y^2 < vf/pi about the RVE centre.
double fibre_fraction(int n, int i, int j, double rad2) {
    int inside = 0;
    for (int b = 0; b < 16; ++b)
        for (int a = 0; a < 16; ++a) {
            const double x = (i + (a + 0.5) / 16.0) / n - 0.5, y = (j + (b + 0.5) / 16.0) / n - 0.5;
            inside += (x * x + y * y < rad2) ? 1 : 0;
        }
    return inside / 256.0;
}

}  // namespace

// -------------------------------------------------------------------------------------------------
extern "C" int ceos_fe2_create(int n_rve, const int* n_cells, const double* vf, double mu_matrix, double stiff_ratio,
                               double k_over_mu, int device, void** handle) {
    if (n_rve < 1 || !n_cells || !vf || !handle) return CEOS_E_ARG;
    Fe2* f = new Fe2();
    *handle = nullptr;
    f->n_rve = n_rve;
    f->device = device;
    // round-off level of the nodal forces of a unit RVE with the stiffer phase
    f->force_floor = 1e-11 * mu_matrix * std::max(1.0, stiff_ratio);
    f->mu_m = mu_matrix;
    f->mu_f = mu_matrix * stiff_ratio;
    f->k_over_mu = k_over_mu;
    f->n.assign(n_cells, n_cells + n_rve);
    f->vf_nominal.assign(vf, vf + n_rve);
    // ---- union mesh: RVE r = unit cube, n^3 cells; fibre along z through the centre ----
    std::vector<double> X;
    std::vector<int> conn, fmap_host, gcoord;
    std::vector<double> eparams;  // [n_elem][2] (Mu, Lambda) of each cell
    const double mu_f = mu_matrix * stiff_ratio;
    f->node_off.assign(n_rve + 1, 0);
    f->red_off.assign(n_rve + 1, 0);
    f->nodes_of.assign(n_rve, 0);
    f->vf_actual.assign(n_rve, 0.0);
    for (int r = 0; r < n_rve; ++r) {
        const int n = f->n[r];
        // the solver keeps 7 FP32 vectors of 3(n^3-1) entries in shared memory: n <= 14 fits
        // the 227 KB a CTA can hold
        if (n < 2 || n > kMaxCells) { delete f; return CEOS_E_ARG; }
        const int m = n + 1;
        const int base = f->node_off[r];
        f->nodes_of[r] = m * m * m;
        f->node_off[r + 1] = base + m * m * m;
        f->red_off[r + 1] = f->red_off[r] + 3 * (n * n * n - 1);
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < m; ++j)
                for (int i = 0; i < m; ++i) {
                    X.push_back((double)i / n);
                    X.push_back((double)j / n);
                    X.push_back((double)k / n);
                    gcoord.push_back(i | (j << 8) | (k << 16));
                    const int ind = (k % n) * n * n + (j % n) * n + (i % n);  // independent node
                    for (int d = 0; d < 3; ++d) fmap_host.push_back(ind == 0 ? -1 : f->red_off[r] + 3 * (ind - 1) + d);
                }
        const double rad2 = vf[r] / M_PI;
        double phisum = 0.0;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    auto id = [&](int a, int b, int c) { return base + (c * m + b) * m + a + 1; };
                    const int e[8] = {id(i, j, k), id(i + 1, j, k), id(i + 1, j + 1, k), id(i, j + 1, k),
                                      id(i, j, k + 1), id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1), id(i, j + 1, k + 1)};
                    conn.insert(conn.end(), e, e + 8);
                    const double phi = fibre_fraction(n, i, j, rad2);
                    phisum += phi;
                    const double mu_e = phi * mu_f + (1.0 - phi) * mu_matrix;
                    const double k_e = phi * (k_over_mu * mu_f) + (1.0 - phi) * (k_over_mu * mu_matrix);
                    eparams.push_back(mu_e);
                    eparams.push_back(k_e - 2.0 * mu_e / 3.0);
                }
        f->vf_actual[r] = phisum / ((double)n * n * n);
    }
    f->n_nodes = f->node_off[n_rve];
    f->n_red = f->red_off[n_rve];
    // ---- element loop: compressible Neo-Hookean cells (ModCompressibleNeoHookean.f90) ----
    ceos_material mat{CEOS_CNH, 1, 2, eparams.data()};
    ceos_mesh mesh{f->n_nodes, (int)(conn.size() / 8), X.data(), conn.data(), nullptr};
    void* lh = nullptr;
    int rc = ceos_create(&mesh, &mat, 1, CEOS_FP64, device, &lh);
    if (rc) { delete f; return rc; }
    f->loop = static_cast<Handle*>(lh);
    f->nnz = f->loop->nnz;
    // ---- device arrays ----
    std::vector<int> rve_of_node(f->n_nodes), rve_of_elem;
    for (int r = 0; r < n_rve; ++r) {
        for (int a = f->node_off[r]; a < f->node_off[r + 1]; ++a) rve_of_node[a] = r;
        rve_of_elem.insert(rve_of_elem.end(), (size_t)f->n[r] * f->n[r] * f->n[r], r);
    }
    std::vector<int> col(f->nnz), rowmap(3 * f->n_nodes + 1);
    ceos_pattern(f->loop, nullptr, nullptr, rowmap.data(), col.data(), nullptr);
    for (auto& c : col) c -= 1;
    std::vector<int> rcol(f->nnz);
    for (long long p = 0; p < f->nnz; ++p) {
        const int g = fmap_host[col[p]];
        rcol[p] = g < 0 ? -1 : g - f->red_off[rve_of_node[col[p] / 3]];
    }
    std::vector<int> order(n_rve);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return f->n[a] > f->n[b]; });
    std::vector<int> ncell(f->n), ones(n_rve, 1);
    const size_t nd = 3 * (size_t)f->n_nodes;
    auto up = [&](void** dst, const void* src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(dst, bytes);
        if (e == cudaSuccess && src) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        return e;
    };
    cudaSetDevice(device);
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up((void**)&f->d_node_off, f->node_off.data(), sizeof(int) * (n_rve + 1));
    if (e == cudaSuccess) e = up((void**)&f->d_red_off, f->red_off.data(), sizeof(int) * (n_rve + 1));
    if (e == cudaSuccess) e = up((void**)&f->d_ncell, ncell.data(), sizeof(int) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_rve_of_node, rve_of_node.data(), sizeof(int) * f->n_nodes);
    if (e == cudaSuccess) e = up((void**)&f->d_fmap, fmap_host.data(), sizeof(int) * nd);
    if (e == cudaSuccess) e = up((void**)&f->d_col, col.data(), sizeof(int) * f->nnz);
    if (e == cudaSuccess) e = up((void**)&f->d_rcol, rcol.data(), sizeof(int) * f->nnz);
    std::vector<int> rve_of_blk(f->n_red / 3);
    for (int r = 0; r < n_rve; ++r)
        for (int q = f->red_off[r] / 3; q < f->red_off[r + 1] / 3; ++q) rve_of_blk[q] = r;
    if (e == cudaSuccess) e = up((void**)&f->d_gcoord, gcoord.data(), sizeof(int) * gcoord.size());
    if (e == cudaSuccess) e = up((void**)&f->d_rve_of_blk, rve_of_blk.data(), sizeof(int) * rve_of_blk.size());
    if (e == cudaSuccess) e = up((void**)&f->d_kell, nullptr, sizeof(float) * 81 * (size_t)f->n_red);
    if (e == cudaSuccess) e = up((void**)&f->d_order, order.data(), sizeof(int) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_queue, nullptr, sizeof(int));
    if (e == cudaSuccess) e = up((void**)&f->d_Fbar, nullptr, sizeof(double) * 9 * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_w, nullptr, sizeof(double) * f->n_red);
    if (e == cudaSuccess) e = up((void**)&f->d_u, nullptr, sizeof(double) * nd);
    if (e == cudaSuccess) e = up((void**)&f->d_rhs, nullptr, sizeof(double) * f->n_red);
    if (e == cudaSuccess) e = up((void**)&f->d_dx, nullptr, sizeof(double) * f->n_red);
    if (e == cudaSuccess) e = up((void**)&f->d_r64, nullptr, sizeof(double) * f->n_red);
    if (e == cudaSuccess) e = up((void**)&f->d_y64, nullptr, sizeof(double) * std::max(nd, (size_t)3 * f->n_red));
    if (e == cudaSuccess) e = up((void**)&f->d_minv, nullptr, sizeof(float) * 9 * (size_t)(f->n_red / 3 + 1));
    if (e == cudaSuccess) e = up((void**)&f->d_rnorm, nullptr, sizeof(double) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_cg_iters, nullptr, sizeof(int) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_active, ones.data(), sizeof(int) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_P, nullptr, sizeof(double) * 9 * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_nn, nullptr, sizeof(double) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_rve_of_elem, rve_of_elem.data(), sizeof(int) * rve_of_elem.size());
    if (e == cudaSuccess) e = up((void**)&f->d_fail, nullptr, sizeof(int) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_op, nullptr, sizeof(int) * n_rve);
    if (e == cudaSuccess) e = up((void**)&f->d_wc, nullptr, sizeof(double) * f->n_red);
    if (e == cudaSuccess) e = up((void**)&f->d_eta, nullptr, sizeof(double) * n_rve);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_Fs, sizeof(double) * 9 * n_rve, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_rn, sizeof(double) * n_rve, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_eta, sizeof(double) * n_rve, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_op, sizeof(int) * n_rve, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_need, sizeof(int) * n_rve, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_cgi, sizeof(int) * n_rve, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&f->hp_status, sizeof(int), cudaHostAllocDefault);
    if (e != cudaSuccess) { delete f; return CEOS_E_CUDA; }
    *handle = f;
    return 0;
}

extern "C" int ceos_fe2_info(void* handle, int* n_nodes, int* n_elem, int* n_red, double* vf_actual) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f) return CEOS_E_ARG;
    if (n_nodes) *n_nodes = f->n_nodes;
    if (n_elem) *n_elem = f->loop->n_elem;
    if (n_red) *n_red = f->n_red;
    if (vf_actual) std::copy(f->vf_actual.begin(), f->vf_actual.end(), vf_actual);
    return 0;
}

extern "C" int ceos_fe2_solve(void* handle, const double* Fbar, double tol, int max_newton, double* P, double* A,
                              int* newton_iters, int* cg_iters) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f || !Fbar || !P || max_newton < 1 || !(tol > 0.0)) return CEOS_E_ARG;
    Handle* h = f->loop;
    cudaStream_t s = h->stream;
    const int nr = f->n_rve;
    CKF(cudaSetDevice(f->device));
    // Start of every RVE's path: Fbar = I with zero fluctuation, or (warm start) the Fbar and
    // fluctuation of its last converged state, which d_w and d_wc both hold after a solve.
    if (!f->warm || f->F_prev.size() != 9 * (size_t)nr) {
        f->F_prev.assign(9 * (size_t)nr, 0.0);
        for (int r = 0; r < nr; ++r) f->F_prev[9 * (size_t)r] = f->F_prev[9 * (size_t)r + 4] = f->F_prev[9 * (size_t)r + 8] = 1.0;
        CKF(cudaMemsetAsync(f->d_w, 0, sizeof(double) * f->n_red, s));
        CKF(cudaMemsetAsync(f->d_wc, 0, sizeof(double) * f->n_red, s));
    }
    const std::vector<double> Fp = f->F_prev;
    CKF(cudaMemsetAsync(f->d_dx, 0, sizeof(double) * f->n_red, s));
    const bool verbose = std::getenv("CEOS_FE2_VERBOSE") != nullptr;
    // Per-RVE load continuation Fbar(a) = Fp + a (Fbar - Fp) (Fp = I, or the last converged Fbar
    // with a warm start): each RVE advances from its last
    // converged level a_done towards 1 in steps da (1/n_sub at first).  A Newton step is accepted
    // when no element folds and the residual grows by at most kGrowth (never beyond kDiverge x the
    // residual at the start of the load step); otherwise it is halved
    // (backtracking line search) up to kMaxHalvings times.  A load step that still fails, or does
    // not converge in max_newton iterations, is cut back: the RVE returns to its converged
    // fluctuations and da shrinks by the golden ratio, as the reference's quasi-static driver
    // cuts back its load steps (ModFEMAnalysis.f90:1136-1374).
    // (kMaxHalvings, kMaxCutbacks, kGrowth, kDiverge, kGolden at file scope; a looser growth test (4x)
    // accepted steps whose linear solves then cost more in total)
    std::vector<int> phase(nr, kNewton), nit(nr, 0), halv(nr, 0), cuts(nr, 0), its(nr, 0), cg_tot(nr, 0);
    std::vector<int> op(nr), need(nr), fail(nr);
    std::vector<double> a_done(nr, 0.0), da(nr, 1.0 / std::max(1, f->n_sub)), a_try(nr), r0(nr, 1.0), racc(nr, 0.0),
        rn(nr), eta(nr, 1.0);
    for (int r = 0; r < nr; ++r) a_try[r] = std::min(1.0, da[r]);
    for (int r = 0; r < nr && !f->solve_mask.empty(); ++r)
        if (!f->solve_mask[r]) {  // skipped: stays at its current state
            phase[r] = kDone;
            a_try[r] = 0.0;
        }
    // every round advances each active RVE by one Newton step, halving, cut-back or load step;
    // a generous cap bounds the whole solve (RVEs still running then fail)
    const int max_rounds = 4 * (max_newton + kMaxHalvings + 2) * (kMaxCutbacks + 2 * std::max(1, f->n_sub) + 8);
    bool all_done = false;
    if (f->device_rounds) {
        // every round on the device: upload the continuation state, one graph launch, read it back
        if (!f->g_rounds) {
            const int rc = build_round_graph(f);
            if (rc) return rc;
        }
        std::vector<int> si(8 * (size_t)nr, 0);
        std::vector<double> sd(6 * (size_t)nr, 0.0);
        for (int r = 0; r < nr; ++r) {
            si[r] = phase[r];
            sd[r] = a_done[r];
            sd[nr + r] = da[r];
            sd[2 * nr + r] = a_try[r];
            sd[3 * nr + r] = r0[r];
            sd[4 * nr + r] = racc[r];
        }
        const double par[4] = {tol, f->force_floor, (double)max_newton, (double)max_rounds};
        int ctl[4] = {0, 0, 0, -1};
        CKF(cudaMemcpyAsync(f->d_rs_int, si.data(), sizeof(int) * si.size(), cudaMemcpyHostToDevice, s));
        CKF(cudaMemcpyAsync(f->d_rs_dbl, sd.data(), sizeof(double) * sd.size(), cudaMemcpyHostToDevice, s));
        CKF(cudaMemcpyAsync(f->d_Fp, Fp.data(), sizeof(double) * 9 * (size_t)nr, cudaMemcpyHostToDevice, s));
        CKF(cudaMemcpyAsync(f->d_Ft, Fbar, sizeof(double) * 9 * (size_t)nr, cudaMemcpyHostToDevice, s));
        CKF(cudaMemcpyAsync(f->d_rpar, par, sizeof(par), cudaMemcpyHostToDevice, s));
        CKF(cudaMemcpyAsync(f->d_rctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, s));
        CKF(cudaGraphLaunch(f->g_rounds, s));
        CKF(cudaMemcpyAsync(si.data(), f->d_rs_int, sizeof(int) * si.size(), cudaMemcpyDeviceToHost, s));
        CKF(cudaMemcpyAsync(sd.data(), f->d_rs_dbl, sizeof(double) * sd.size(), cudaMemcpyDeviceToHost, s));
        CKF(cudaMemcpyAsync(ctl, f->d_rctl, sizeof(ctl), cudaMemcpyDeviceToHost, s));
        CKF(cudaStreamSynchronize(s));
        h->evaluated = true;
        all_done = true;
        for (int r = 0; r < nr; ++r) {
            phase[r] = si[r];
            its[r] = si[4 * nr + r];
            cg_tot[r] = si[5 * nr + r];
            a_done[r] = sd[r];
            if (phase[r] == kNewton) all_done = false;
        }
        if (ctl[2]) {
            f->msg = "RVE " + std::to_string(ctl[3]) + ": no convergence after " + std::to_string(kMaxCutbacks) +
                     " load cut-backs (converged load level " + std::to_string(a_done[ctl[3]]) + ")";
            return 1;
        }
        if (verbose) std::fprintf(stderr, "fe2: %d device-resident rounds\n", ctl[0]);
    }
    for (int round = 0; !f->device_rounds && round < max_rounds && !all_done; ++round) {
        for (int r = 0; r < nr; ++r)
            for (int k = 0; k < 9; ++k) {
                const size_t i = 9 * (size_t)r + k;
                f->hp_Fs[i] = Fp[i] + a_try[r] * (Fbar[i] - Fp[i]);
            }
        int rc = f->g_assemble ? 0 : capture(f, record_assemble, &f->g_assemble);
        if (rc) return rc;
        CKF(cudaGraphLaunch(f->g_assemble, s));
        CKF(cudaStreamSynchronize(s));
        h->evaluated = true;
        int st = 0;
        if (*f->hp_status) {
            st = ceos_status(h, nullptr);
            if (st < 0) return st;
        }
        std::fill(fail.begin(), fail.end(), 0);
        if (st) {
            CKF(cudaMemsetAsync(f->d_fail, 0, sizeof(int) * nr, s));
            rve_fail_kernel<<<(h->n_elem + 255) / 256, 256, 0, s>>>(h->n_elem, h->d_elem_status, f->d_rve_of_elem,
                                                                    f->d_fail);
            CKF(cudaGetLastError());
            CKF(cudaMemcpyAsync(fail.data(), f->d_fail, sizeof(int) * nr, cudaMemcpyDeviceToHost, s));
            CKF(cudaStreamSynchronize(s));
        }
        std::copy(f->hp_rn, f->hp_rn + nr, rn.begin());
        all_done = true;
        int n_need = 0, n_rej = 0, n_cut = 0;
        double worst = 0.0;
        for (int r = 0; r < nr; ++r) {
            op[r] = kOpNone;
            need[r] = 0;
            if (phase[r] != kNewton) continue;
            all_done = false;
            RveCont c{phase[r], nit[r], halv[r], cuts[r], its[r], a_done[r], da[r], a_try[r], r0[r], racc[r]};
            const int flags = decide_rve(c, rn[r], !fail[r] && std::isfinite(rn[r]), tol, f->force_floor, max_newton,
                                         op[r], need[r], eta[r]);
            phase[r] = c.phase;
            nit[r] = c.nit;
            halv[r] = c.halv;
            cuts[r] = c.cuts;
            its[r] = c.its;
            a_done[r] = c.a_done;
            da[r] = c.da;
            a_try[r] = c.a_try;
            r0[r] = c.r0;
            racc[r] = c.racc;
            if (flags & kExhausted) {
                f->msg = "RVE " + std::to_string(r) + ": no convergence after " + std::to_string(kMaxCutbacks) +
                         " load cut-backs (converged load level " + std::to_string(a_done[r]) + ")";
                if (!f->allow_failures) return st ? st : 1;
            }
            n_rej += (flags & kRejected) ? 1 : 0;
            n_cut += (flags & kCut) ? 1 : 0;
            if (need[r]) {
                ++n_need;
                worst = std::max(worst, rn[r] / r0[r]);
            }
        }
        if (verbose)
            std::fprintf(stderr, "fe2: round %d solving %d max rel residual %.3e rejected %d cut back %d\n", round,
                         n_need, worst, n_rej, n_cut);
        if (all_done) break;
        std::copy(op.begin(), op.end(), f->hp_op);
        if (n_need) {
            std::copy(need.begin(), need.end(), f->hp_need);
            std::copy(eta.begin(), eta.end(), f->hp_eta);
            rc = f->g_solve ? 0 : capture(f, record_solve, &f->g_solve);
            if (rc) return rc;
            CKF(cudaGraphLaunch(f->g_solve, s));
            CKF(cudaStreamSynchronize(s));
            for (int r = 0; r < nr; ++r)
                if (need[r]) cg_tot[r] += f->hp_cgi[r];
        } else {
            CKF(cudaMemcpyAsync(f->d_op, f->hp_op, sizeof(int) * nr, cudaMemcpyHostToDevice, s));
            rve_op_kernel<<<nr, 256, 0, s>>>(nr, f->d_red_off, f->d_op, f->d_w, f->d_dx, f->d_wc);
            CKF(cudaGetLastError());
        }
    }
    if (!all_done) {
        f->msg = "load continuation did not finish";
        if (!f->allow_failures) return 1;
        for (int r = 0; r < nr; ++r)
            if (phase[r] == kNewton) phase[r] = kFailed;  // the last assembly is not at their converged state
    }
    int n_failed = 0;
    for (int r = 0; r < nr; ++r) {
        if (phase[r] == kFailed) {
            ++n_failed;
            its[r] = -1;
        }
        for (int k = 0; k < 9; ++k) {  // the converged state each RVE ends in (partial for failed ones)
            const size_t i = 9 * (size_t)r + k;
            f->F_prev[i] = Fp[i] + a_done[r] * (Fbar[i] - Fp[i]);
        }
    }
    if (n_failed) f->msg = std::to_string(n_failed) + " RVE(s) did not converge";
    // converged state: K and f_int of the last assembly
    homogenize_kernel<<<f->n_rve, 256, 0, s>>>(f->n_rve, f->d_node_off, h->d_X, h->d_fint, f->d_P, 1.0);
    CKF(cudaGetLastError());
    CKF(cudaMemcpyAsync(P, f->d_P, sizeof(double) * 9 * f->n_rve, cudaMemcpyDeviceToHost, s));
    if (A) {
        // static condensation with the 9 affine modes
        const size_t nd = 3 * (size_t)f->n_nodes;
        if (!f->d_Z) {
            CKF(cudaMalloc(&f->d_A, sizeof(double) * 81 * f->n_rve));
            CKF(cudaMalloc(&f->d_Z, sizeof(double) * 81 * f->n_rve));
            CKF(cudaMalloc(&f->d_M, sizeof(double) * 9 * (size_t)f->n_red));
            CKF(cudaMalloc(&f->d_X9, sizeof(double) * 9 * (size_t)f->n_red));
        }
        for (int kL = 0; kL < 9; ++kL) {
            affine_mode_kernel<<<(int)((nd + 255) / 256), 256, 0, s>>>(f->n_nodes, h->d_X, kL, f->d_u);
            CKF(cudaMemsetAsync(f->d_y64, 0, sizeof(double) * nd, s));
            spmv_upper_kernel<<<(int)((nd * 32 + 255) / 256), 256, 0, s>>>((int)nd, h->d_rs, h->d_nup, f->d_col,
                                                                         h->d_kval, f->d_u, f->d_y64);
            zkz_kernel<<<f->n_rve, 256, 0, s>>>(f->n_rve, f->d_node_off, h->d_X, f->d_y64, kL, f->d_Z, 1.0);
            CKF(cudaMemsetAsync(f->d_M + (size_t)kL * f->n_red, 0, sizeof(double) * f->n_red, s));
            fold_kernel<<<(int)((nd + 255) / 256), 256, 0, s>>>((int)nd, f->d_fmap, f->d_y64, f->d_M + (size_t)kL * f->n_red,
                                                               1.0);
            CKF(cudaGetLastError());
        }
        std::vector<int> ones(f->n_rve, 1);  // masked-out RVEs need no new tangent either
        if (!f->solve_mask.empty()) ones = f->solve_mask;
        std::vector<double> eta_t(f->n_rve, 1e-8);
        CKF(cudaMemcpyAsync(f->d_active, ones.data(), sizeof(int) * f->n_rve, cudaMemcpyHostToDevice, s));
        CKF(cudaMemcpyAsync(f->d_eta, eta_t.data(), sizeof(double) * f->n_rve, cudaMemcpyHostToDevice, s));
        int rc = run_solver(f, 9, f->d_M, f->d_X9, 4000, 8);
        if (rc) return rc;
        condense_kernel<<<f->n_rve, 256, 0, s>>>(f->n_rve, f->d_red_off, f->n_red, f->d_M, f->d_X9, f->d_Z, f->d_A, 1.0);
        CKF(cudaGetLastError());
        CKF(cudaMemcpyAsync(A, f->d_A, sizeof(double) * 81 * f->n_rve, cudaMemcpyDeviceToHost, s));
    }
    CKF(cudaStreamSynchronize(s));
    for (int r = 0; r < nr; ++r)
        if (phase[r] == kFailed) {
            for (int k = 0; k < 9; ++k) P[9 * (size_t)r + k] = std::nan("");
            if (A)
                for (int k = 0; k < 81; ++k) A[81 * (size_t)r + k] = std::nan("");
        }
    if (newton_iters) std::copy(its.begin(), its.end(), newton_iters);
    if (cg_iters) std::copy(cg_tot.begin(), cg_tot.end(), cg_iters);
    return n_failed ? 2 : 0;
}

// Warm start: every solve continues each RVE from the Fbar and fluctuation of its last converged
// state (an FE^2 macro iteration moves Fbar a little; the RVE follows the macro load path instead
// of restarting from the undeformed state).
extern "C" int ceos_fe2_set_warm_start(void* handle, int on) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f) return CEOS_E_ARG;
    f->warm = on ? 1 : 0;
    return 0;
}

// mask [n_rve]: 0 = leave the RVE out of the next solves (it keeps its state, P is that of the state,
// its tangent rows are not recomputed); NULL = solve all.
extern "C" int ceos_fe2_set_solve_mask(void* handle, const int* mask) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f) return CEOS_E_ARG;
    if (mask) f->solve_mask.assign(mask, mask + f->n_rve);
    else f->solve_mask.clear();
    return 0;
}

// Number of RVEs the persistent MINRES kernel keeps in flight (0: automatic, bounded by the L2 size).
extern "C" int ceos_fe2_set_solver_ctas(void* handle, int n) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f || n < 0) return CEOS_E_ARG;
    f->solver_ctas = n;
    f->drop_graphs();  // the solve graph holds the launch shape
    return 0;
}

// Autotuner of the MINRES launch shape (threads per RVE x RVEs in flight): assembles the first
// Newton system of every RVE at Fbar (row-major [n_rve][9]) from its current fluctuations, times
// the linear solve of that system (Newton forcing 1e-2, the typical first tolerance) once per
// candidate with CUDA events, keeps the fastest shape and reports it.  The fluctuations are not
// changed.  ms_out (n_cand entries, or NULL) receives the times in the order threads {256, 512}
// x RVEs in flight {occupancy limit, 2 per SM, 1 per SM}; candidates that coincide report -1.
extern "C" int ceos_fe2_autotune(void* handle, const double* Fbar, int* threads, int* ctas, double* ms_out,
                                 int n_cand) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f || !Fbar) return CEOS_E_ARG;
    Handle* h = f->loop;
    cudaStream_t s = h->stream;
    const int nr = f->n_rve;
    CKF(cudaSetDevice(f->device));
    std::copy(Fbar, Fbar + 9 * (size_t)nr, f->hp_Fs);
    f->drop_graphs();
    int rc = record_assemble(f);
    if (rc) return rc;
    for (int r = 0; r < nr; ++r) {
        f->hp_need[r] = 1;
        f->hp_eta[r] = 1e-2;
    }
    CKF(cudaMemcpyAsync(f->d_active, f->hp_need, sizeof(int) * nr, cudaMemcpyHostToDevice, s));
    CKF(cudaMemcpyAsync(f->d_eta, f->hp_eta, sizeof(double) * nr, cudaMemcpyHostToDevice, s));
    int max_m = 0;
    for (int r = 0; r < nr; ++r) max_m = std::max(max_m, f->red_off[r + 1] - f->red_off[r]);
    const size_t smem = solve_smem_bytes(max_m);
    CKF(cudaFuncSetAttribute(fe2_minres_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device);
    cudaEvent_t e0, e1;
    CKF(cudaEventCreate(&e0));
    CKF(cudaEventCreate(&e1));
    const int keep_threads = f->solver_threads, keep_ctas = f->solver_ctas;
    int best_t = keep_threads, best_c = keep_ctas, k = 0;
    float best_ms = -1.f;
    std::vector<long long> seen;
    for (int bs : {256, 512}) {
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fe2_minres_kernel, bs, smem);
        const int full = std::max(1, std::min(nr, sms * std::max(per_sm, 1)));
        for (int c : {0, 2 * sms, sms}) {
            const int grid = c == 0 ? full : std::max(1, std::min(full, c));
            const long long key = (long long)bs << 32 | grid;
            float ms = -1.f;
            if (std::find(seen.begin(), seen.end(), key) == seen.end()) {
                seen.push_back(key);
                f->solver_threads = bs;
                f->solver_ctas = c == 0 ? 0 : grid;
                CKF(cudaMemsetAsync(f->d_dx, 0, sizeof(double) * f->n_red, s));
                CKF(cudaEventRecord(e0, s));
                rc = run_solver(f, 1, f->d_rhs, f->d_dx, 2000, 3);
                if (rc) break;
                CKF(cudaEventRecord(e1, s));
                CKF(cudaEventSynchronize(e1));
                CKF(cudaEventElapsedTime(&ms, e0, e1));
                if (best_ms < 0.f || ms < best_ms) {
                    best_ms = ms;
                    best_t = bs;
                    best_c = f->solver_ctas;
                }
            }
            if (ms_out && k < n_cand) ms_out[k] = ms;
            ++k;
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CKF(cudaMemsetAsync(f->d_dx, 0, sizeof(double) * f->n_red, s));
    CKF(cudaStreamSynchronize(s));
    if (rc) {
        f->solver_threads = keep_threads;
        f->solver_ctas = keep_ctas;
        return rc;
    }
    f->solver_threads = best_t;
    f->solver_ctas = best_c;
    if (threads) *threads = best_t;
    if (ctas) *ctas = best_c;
    return 0;
}

// Report RVEs that cannot converge (P and A set to NaN, newton_iters -1, return value 2) instead of
// failing the whole solve.
extern "C" int ceos_fe2_set_allow_failures(void* handle, int allow) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f) return CEOS_E_ARG;
    if ((allow ? 1 : 0) != f->allow_failures && f->g_rounds) {  // the round graph holds the flag
        cudaGraphExecDestroy(f->g_rounds);
        f->g_rounds = nullptr;
    }
    f->allow_failures = allow ? 1 : 0;
    return 0;
}

extern "C" int ceos_fe2_set_device_rounds(void* handle, int on) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f) return CEOS_E_ARG;
    f->device_rounds = on ? 1 : 0;
    return 0;
}

// New fibre volume fractions for the same RVE sizes (cell moduli recomputed, mesh kept); RVEs whose
// fraction changes restart from the undeformed state at the next solve.
extern "C" int ceos_fe2_set_fractions(void* handle, const double* vf) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f || !vf) return CEOS_E_ARG;
    f->drop_graphs();
    std::vector<double> eparams;
    eparams.reserve(2 * (size_t)f->loop->n_elem);
    std::vector<int> changed(f->n_rve, 0);
    for (int r = 0; r < f->n_rve; ++r) {
        const int n = f->n[r];
        changed[r] = vf[r] != f->vf_nominal[r];
        const double rad2 = vf[r] / M_PI;
        double phisum = 0.0;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    const double phi = fibre_fraction(n, i, j, rad2);
                    phisum += phi;
                    const double mu_e = phi * f->mu_f + (1.0 - phi) * f->mu_m;
                    const double k_e = phi * (f->k_over_mu * f->mu_f) + (1.0 - phi) * (f->k_over_mu * f->mu_m);
                    eparams.push_back(mu_e);
                    eparams.push_back(k_e - 2.0 * mu_e / 3.0);
                }
        f->vf_nominal[r] = vf[r];
        f->vf_actual[r] = phisum / ((double)n * n * n);
    }
    // RVEs with a new fraction restart from the undeformed state; the others keep their warm state
    if (f->F_prev.size() == 9 * (size_t)f->n_rve) {
        Handle* h = f->loop;
        for (int r = 0; r < f->n_rve; ++r) {
            if (!changed[r]) continue;
            for (int k = 0; k < 9; ++k) f->F_prev[9 * (size_t)r + k] = (k % 4 == 0) ? 1.0 : 0.0;
            const size_t q0 = f->red_off[r], m = f->red_off[r + 1] - f->red_off[r];
            CKF(cudaMemsetAsync(f->d_w + q0, 0, sizeof(double) * m, h->stream));
            CKF(cudaMemsetAsync(f->d_wc + q0, 0, sizeof(double) * m, h->stream));
        }
    }
    return ceos_update_params(f->loop, eparams.data());
}

extern "C" int ceos_fe2_set_increments(void* handle, int n_sub) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f || n_sub < 1) return CEOS_E_ARG;
    f->n_sub = n_sub;
    return 0;
}

extern "C" int ceos_fe2_message(void* handle, char* msg, int msg_len) {
    Fe2* f = static_cast<Fe2*>(handle);
    if (!f || !msg || msg_len < 1) return CEOS_E_ARG;
    std::snprintf(msg, msg_len, "%s", f->msg.c_str());
    return 0;
}

extern "C" void ceos_fe2_destroy(void* handle) { delete static_cast<Fe2*>(handle); }
