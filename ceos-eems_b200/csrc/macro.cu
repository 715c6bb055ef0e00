// macro.cu -- device linear solver for the Newton iteration of a macro (or any) mesh, and a state
// scatter for Gauss points whose response comes from RVE solves.
//
// The reference hands the assembled upper-CSR system to PARDISO on the host
// (FEM/Modules/ModFEMSystemOfEquations.f90, Tools/MathTools/ModNewtonRaphsonFull.f90:44-168, with
// the Dirichlet rows of ApplyBoundaryConditionsNEW, ModBoundaryConditions.f90:246-340).  Here the
// system stays on the device: block-Jacobi (3x3 nodal) preconditioned CG on the symmetric matrix
// stored as the element loop's upper CSR, prescribed dofs eliminated by masking (their rows and
// columns act as identity, their correction is zero).  Every scalar of the recurrence lives in
// device memory, so a block of iterations is one CUDA graph replay with no host round trip;
// the host checks the residual between blocks.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ceos_gpu.h"
#include "ceos_handle.h"

namespace {

using ceos::Handle;
constexpr int kIterPerGraph = 16;

struct Pcg {
    Handle* h = nullptr;
    int n_dof = 0, n_nodes = 0;
    cudaStream_t stream = nullptr;
    double *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    float* minv = nullptr;    // [n_nodes][9]
    double* sc = nullptr;     // [0] rz, [1] pq, [2] rz_new, [3] rr, [4] rr0
    double* hist = nullptr;   // [kIterPerGraph] rr after each iteration of the last block
    int* col1 = nullptr;      // [nnz] 1-based CSR columns of the loop's pattern
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const double* gK = nullptr;       // operands the captured graph was built for
    const uint8_t* gfix = nullptr;
    double* gx = nullptr;
    std::string msg;
    ~Pcg() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        void* ptrs[] = {r, z, p, q, minv, sc, hist, col1};
        for (void* v : ptrs)
            if (v) cudaFree(v);
        if (stream) cudaStreamDestroy(stream);
    }
};

__device__ __forceinline__ long long row_start(const long long* rs, const int* nup, int row, int* len) {
    const int a = row / 3, k = row - 3 * a, m = nup[a];
    *len = (3 - k) + 3 * m;
    return rs[a] + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
}

// y = K_ff p over free dofs (p is zero on prescribed dofs); warp per row, transposed half by atomics
__global__ void spmv_kernel(int n_dof, const long long* rs, const int* nup, const int* col1, const double* K,
                            const uint8_t* fix, const double* p, double* y) {
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= n_dof || fix[row]) return;
    int len;
    const long long start = row_start(rs, nup, row, &len);
    const double pr = p[row];
    double acc = 0.0;
    for (int t = lane; t < len; t += 32) {
        const int c = col1[start + t] - 1;
        if (fix[c]) continue;
        const double v = K[start + t];
        acc += v * p[c];
        if (c != row) atomicAdd(y + c, v * pr);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) atomicAdd(y + row, acc);
}

__device__ __forceinline__ void block_add(double v, double* dst) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
}

// SPD block-Jacobi inverse per node on the free dofs (prescribed rows/cols -> identity)
__global__ void pcg_blocks_kernel(int n_nodes, const long long* rs, const int* nup, const double* K,
                                  const uint8_t* fix, float* minv) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_nodes) return;
    const long long r0 = rs[a];
    const int m = nup[a];
    const long long r1 = r0 + 3 + 3LL * m, r2 = r1 + 2 + 3LL * m;
    double A[9] = {K[r0], K[r0 + 1], K[r0 + 2], K[r0 + 1], K[r1], K[r1 + 1], K[r0 + 2], K[r1 + 1], K[r2]};
    for (int d = 0; d < 3; ++d)
        if (fix[3 * a + d])
            for (int k = 0; k < 3; ++k) {
                A[3 * d + k] = (k == d) ? 1.0 : 0.0;
                A[3 * k + d] = (k == d) ? 1.0 : 0.0;
            }
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
    const bool pd = A[0] > 0.0 && c[8] > 1e-12 * A[0] * A[4] && det > 1e-12 * A[0] * A[4] * A[8];
    float* M = minv + 9 * (size_t)a;
    if (pd) {
        for (int k = 0; k < 9; ++k) M[k] = (float)(c[k] / det);
    } else {
        for (int k = 0; k < 9; ++k) M[k] = 0.f;
        for (int d = 0; d < 3; ++d) M[4 * d] = (float)(1.0 / fmax(fabs(A[4 * d]), 1e-300));
    }
}

__device__ __forceinline__ void apply_minv(const float* M, const double r[3], double z[3]) {
    for (int i = 0; i < 3; ++i) z[i] = (double)M[3 * i] * r[0] + (double)M[3 * i + 1] * r[1] + (double)M[3 * i + 2] * r[2];
}

// x = 0, r = b (zero on prescribed dofs), z = M r, p = z, rz, rr
__global__ void pcg_init_kernel(int n_nodes, const uint8_t* fix, const float* minv, const double* b, double* x,
                                double* r, double* z, double* p, double* sc) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double rz = 0.0, rr = 0.0;
    if (a < n_nodes) {
        double rv[3], zv[3];
        for (int d = 0; d < 3; ++d) rv[d] = fix[3 * a + d] ? 0.0 : b[3 * a + d];
        apply_minv(minv + 9 * (size_t)a, rv, zv);
        for (int d = 0; d < 3; ++d) {
            if (fix[3 * a + d]) zv[d] = 0.0;
            x[3 * a + d] = 0.0;
            r[3 * a + d] = rv[d];
            z[3 * a + d] = zv[d];
            p[3 * a + d] = zv[d];
            rz += rv[d] * zv[d];
            rr += rv[d] * rv[d];
        }
    }
    block_add(rz, sc + 0);
    block_add(rr, sc + 4);
}

__global__ void pcg_dot_kernel(int n, const double* a, const double* b, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    block_add(i < n ? a[i] * b[i] : 0.0, out);
}

// alpha = rz / pq; x += alpha p; r -= alpha q; z = M r; accumulate rz_new and rr
__global__ void pcg_update_kernel(int n_nodes, const uint8_t* fix, const float* minv, double* x, double* r, double* z,
                                  const double* p, const double* q, double* sc) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const double alpha = sc[1] != 0.0 ? sc[0] / sc[1] : 0.0;
    double rz = 0.0, rr = 0.0;
    if (a < n_nodes) {
        double rv[3], zv[3];
        for (int d = 0; d < 3; ++d) {
            const int i = 3 * a + d;
            x[i] += alpha * p[i];
            rv[d] = fix[i] ? 0.0 : r[i] - alpha * q[i];
            r[i] = rv[d];
        }
        apply_minv(minv + 9 * (size_t)a, rv, zv);
        for (int d = 0; d < 3; ++d) {
            const int i = 3 * a + d;
            if (fix[i]) zv[d] = 0.0;
            z[i] = zv[d];
            rz += rv[d] * zv[d];
            rr += rv[d] * rv[d];
        }
    }
    block_add(rz, sc + 2);
    block_add(rr, sc + 3);
}

__global__ void pcg_direction_kernel(int n, const double* z, double* p, const double* sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double beta = sc[0] != 0.0 ? sc[2] / sc[0] : 0.0;
    if (i < n) p[i] = z[i] + beta * p[i];
}

// rz <- rz_new, record rr, clear the accumulators
__global__ void pcg_scalars_kernel(double* sc, double* hist, int k) {
    hist[k] = sc[3];
    sc[0] = sc[2];
    sc[1] = sc[2] = sc[3] = 0.0;
}

// state[(v*8 + gp)*ld + e] = vals[i][v] for points q_i = gp * n_elem + e
template <typename T>
__global__ void scatter_state_kernel(int n_pts, int nv, const int* q, const double* vals, int n_elem, long long ld,
                                     T* state) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pts) return;
    const int gp = q[i] / n_elem, e = q[i] - gp * n_elem;
    for (int v = 0; v < nv; ++v) state[((size_t)v * 8 + gp) * ld + e] = (T)vals[(size_t)i * nv + v];
}

#define CKP(call)                                                              \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            g->msg = std::string(#call) + ": " + cudaGetErrorString(e_);       \
            return CEOS_E_CUDA;                                                \
        }                                                                      \
    } while (0)

int capture_block(Pcg* g, const double* K, const uint8_t* fix, double* x, const int* col1) {
    Handle* h = g->h;
    cudaStream_t s = g->stream;
    if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
    if (g->graph) { cudaGraphDestroy(g->graph); g->graph = nullptr; }
    CKP(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int nd = g->n_dof, nn = g->n_nodes;
    for (int k = 0; k < kIterPerGraph; ++k) {
        cudaMemsetAsync(g->q, 0, sizeof(double) * nd, s);
        spmv_kernel<<<(unsigned)(((long long)nd * 32 + 255) / 256), 256, 0, s>>>(nd, h->d_rs, h->d_nup, col1, K, fix,
                                                                                  g->p, g->q);
        pcg_dot_kernel<<<(nd + 255) / 256, 256, 0, s>>>(nd, g->p, g->q, g->sc + 1);
        pcg_update_kernel<<<(nn + 127) / 128, 128, 0, s>>>(nn, fix, g->minv, x, g->r, g->z, g->p, g->q, g->sc);
        pcg_direction_kernel<<<(nd + 255) / 256, 256, 0, s>>>(nd, g->z, g->p, g->sc);
        pcg_scalars_kernel<<<1, 1, 0, s>>>(g->sc, g->hist, k);
    }
    const cudaError_t e = cudaStreamEndCapture(s, &g->graph);
    if (e != cudaSuccess) { g->msg = "pcg capture"; return CEOS_E_CUDA; }
    CKP(cudaGraphInstantiate(&g->exec, g->graph, 0));
    g->gK = K;
    g->gfix = fix;
    g->gx = x;
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
extern "C" int ceos_pcg_create(void* loop_handle, void** pcg) {
    Handle* h = static_cast<Handle*>(loop_handle);
    if (!h || !pcg) return CEOS_E_ARG;
    *pcg = nullptr;
    Pcg* g = new Pcg();
    g->h = h;
    g->n_nodes = h->n_nodes;
    g->n_dof = 3 * h->n_nodes;
    bool ok = cudaSetDevice(h->device) == cudaSuccess &&
              cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) == cudaSuccess;
    auto al = [&](void** p, size_t b) { if (ok) ok = cudaMalloc(p, b) == cudaSuccess; };
    al((void**)&g->r, sizeof(double) * g->n_dof);
    al((void**)&g->z, sizeof(double) * g->n_dof);
    al((void**)&g->p, sizeof(double) * g->n_dof);
    al((void**)&g->q, sizeof(double) * g->n_dof);
    al((void**)&g->minv, sizeof(float) * 9 * (size_t)g->n_nodes);
    al((void**)&g->sc, sizeof(double) * 8);
    al((void**)&g->hist, sizeof(double) * kIterPerGraph);
    al((void**)&g->col1, sizeof(int) * h->nnz);
    if (ok) {
        std::vector<int> rowmap(3 * (size_t)h->n_nodes + 1), col(h->nnz);
        ok = ceos_pattern(h, nullptr, nullptr, rowmap.data(), col.data(), nullptr) == 0 &&
             cudaMemcpy(g->col1, col.data(), sizeof(int) * h->nnz, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    if (!ok) { delete g; return CEOS_E_CUDA; }
    *pcg = g;
    return 0;
}

// Solve K_ff x_f = b_f (x = 0 on dofs with fixed[i] != 0) for the element loop's upper CSR K
// (device pointer, FP64), to ||r|| <= tol ||b_f||.  All pointers are device pointers.
// iters / rel_res (host) receive the iteration count and the final relative residual.
extern "C" int ceos_pcg_solve(void* pcg, const double* dK, const unsigned char* dfixed, const double* db, double* dx,
                              double tol, int max_iter, int* iters, double* rel_res) {
    Pcg* g = static_cast<Pcg*>(pcg);
    if (!g || !dK || !dfixed || !db || !dx || max_iter < 1) return CEOS_E_ARG;
    Handle* h = g->h;
    cudaStream_t s = g->stream;
    CKP(cudaSetDevice(h->device));
    CKP(cudaDeviceSynchronize());  // K, b from any stream are complete
    CKP(cudaMemsetAsync(g->sc, 0, sizeof(double) * 8, s));
    pcg_blocks_kernel<<<(g->n_nodes + 127) / 128, 128, 0, s>>>(g->n_nodes, h->d_rs, h->d_nup, dK, dfixed, g->minv);
    pcg_init_kernel<<<(g->n_nodes + 127) / 128, 128, 0, s>>>(g->n_nodes, dfixed, g->minv, db, dx, g->r, g->z, g->p,
                                                            g->sc);
    CKP(cudaGetLastError());
    if (!g->exec || g->gK != dK || g->gfix != dfixed || g->gx != dx) {
        int rc = capture_block(g, dK, dfixed, dx, g->col1);
        if (rc) return rc;
    }
    double rr0 = 0.0;
    CKP(cudaMemcpyAsync(&rr0, g->sc + 4, sizeof(double), cudaMemcpyDeviceToHost, s));
    CKP(cudaStreamSynchronize(s));
    int it = 0;
    double rel = rr0 > 0.0 ? 1.0 : 0.0;
    std::vector<double> hist(kIterPerGraph);
    while (rr0 > 0.0 && it < max_iter && rel > tol) {
        CKP(cudaGraphLaunch(g->exec, s));
        CKP(cudaMemcpyAsync(hist.data(), g->hist, sizeof(double) * kIterPerGraph, cudaMemcpyDeviceToHost, s));
        CKP(cudaStreamSynchronize(s));
        for (int k = 0; k < kIterPerGraph; ++k) {
            ++it;
            rel = std::sqrt(std::max(hist[k], 0.0) / rr0);
            if (rel <= tol) break;
        }
        if (!std::isfinite(rel)) { g->msg = "pcg breakdown"; return CEOS_E_SOLVER; }
    }
    if (iters) *iters = it;
    if (rel_res) *rel_res = rel;
    return rel <= tol ? 0 : CEOS_E_SOLVER;
}

extern "C" void ceos_pcg_destroy(void* pcg) { delete static_cast<Pcg*>(pcg); }

// Write nv values per point into the Gauss-point state of an element loop (committed buffer):
// q [n_pts] point ids (gp * n_elem + e), vals [n_pts][nv] (host arrays).
extern "C" int ceos_state_scatter(void* loop_handle, int n_pts, const int* q, const double* vals, int nv) {
    Handle* h = static_cast<Handle*>(loop_handle);
    if (!h || n_pts < 0 || (n_pts && (!q || !vals)) || nv < 1 || nv > h->nstate) return CEOS_E_ARG;
    if (!n_pts) return 0;
    for (int i = 0; i < n_pts; ++i)
        if (q[i] < 0 || q[i] >= 8 * h->n_elem) return CEOS_E_ARG;
    if (cudaSetDevice(h->device) != cudaSuccess) return CEOS_E_CUDA;
    int* dq = nullptr;
    double* dv = nullptr;
    if (cudaMalloc(&dq, sizeof(int) * n_pts) != cudaSuccess) return CEOS_E_CUDA;
    if (cudaMalloc(&dv, sizeof(double) * nv * (size_t)n_pts) != cudaSuccess) { cudaFree(dq); return CEOS_E_CUDA; }
    cudaMemcpyAsync(dq, q, sizeof(int) * n_pts, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(dv, vals, sizeof(double) * nv * (size_t)n_pts, cudaMemcpyHostToDevice, h->stream);
    void* st = h->d_state[h->cur_old];
    if (h->precision == CEOS_MIXED)
        scatter_state_kernel<float><<<(n_pts + 255) / 256, 256, 0, h->stream>>>(n_pts, nv, dq, dv, h->n_elem, h->ld,
                                                                                static_cast<float*>(st));
    else
        scatter_state_kernel<double><<<(n_pts + 255) / 256, 256, 0, h->stream>>>(n_pts, nv, dq, dv, h->n_elem, h->ld,
                                                                                 static_cast<double*>(st));
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(dq);
    cudaFree(dv);
    return e == cudaSuccess ? 0 : CEOS_E_CUDA;
}
