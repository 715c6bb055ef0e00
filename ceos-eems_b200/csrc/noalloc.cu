// noalloc.cu -- element loop entry point that performs no device allocation.
//
// Some hosts cannot call cudaMalloc when they assemble: their GPU memory is owned by another
// allocator (a host application that reserves the device through its own memory pool, or a
// runtime that forbids new allocations once its solver is running), so every device buffer
// they hand us is theirs.  ceos_cnh_assemble_noalloc serves them: it takes only caller-owned
// device buffers (mesh, CSR pattern, displacements, outputs) and draws the assembly scratch
// from kAsmScratch, a fixed static array in this file, instead of allocating.
//
// The scratch is the FP32 node-pair block accumulator of the blocked assembly (3 rows x 4
// floats per node pair, 48 bytes).  Its size, kAsmScratchBytes = 8 MiB, limits a call to
// 174,762 node-pair blocks (about 12,000 nodes of a structured Hexa8 mesh); larger meshes are
// rejected with CEOS_E_ARG.  Every GPU that loads this library keeps the 8 MiB until the
// process exits.  All calls share the array and it keeps the last call's contents, so each
// call clears the part it uses before accumulating; two calls whose work overlaps on the GPU
// (different streams, or different host threads without ordering) race on it and must not
// be issued.
//
// The kernels keep no per-thread arrays in local memory (ptxas reports a 0-byte stack frame
// for both), so a launch never makes the driver enlarge the context's local-memory reservation,
// which would be a device allocation behind the caller's back.  Per-element data lives in
// static shared memory: a CTA of 128 threads works on 16 elements, thread (element, j) with j
// the Gauss point in the constitutive phase and the node in the assembly phase.
//
// Every index that comes from the caller is checked before it is used: node ids against
// n_nodes, each CSR row triple against the layout of the upper pattern (row 3n holds 3 + 3m
// entries, rows 3n+1 and 3n+2 two and one fewer diagonal entries) and against nnz, and every
// node-pair block against the number of blocks the call cleared.  A failed check skips the
// access and sets a flag; the call then returns CEOS_E_MESH.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/ceos_gpu.h"
#include "ceos_common.cuh"
#include "materials.cuh"

namespace {

constexpr size_t kAsmScratchBytes = 8u << 20;
constexpr long long kAsmScratchBlocks = (long long)(kAsmScratchBytes / 48);

static __device__ __align__(256) float kAsmScratch[kAsmScratchBytes / sizeof(float)];

// Device address of kAsmScratch, resolved once per device with that device current.
constexpr int kMaxDevices = 64;
float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_on_current_device(float** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CEOS_E_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, kAsmScratch) != cudaSuccess || !p) return CEOS_E_CUDA;
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_addr[dev];
    return 0;
}

constexpr int kBadGeometry = 1;  // det J <= 1e-13 (ClassStatus error 1)
constexpr int kBadMesh = 2;      // node id, CSR row or node pair inconsistent with the pattern

__device__ __forceinline__ void red_v4_na(float* p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

// The three CSR rows of node n as the 1-based upper pattern lays them out: row 3n starts at
// rowmap[3n]-1 with 3 + 3m entries (m upper neighbours), row 3n+1 has 2 + 3m, row 3n+2 1 + 3m.
// The node's node-pair blocks start at block n + (r0 - 6n)/9 (one diagonal block per node and
// one per upper neighbour of every earlier node).  ok is false when the rows do not have that
// shape, leave [0, nnz), or their blocks leave [0, n_blocks).
struct NodeRows {
    long long r0, bb;
    int m;
    bool ok;
};
__device__ __forceinline__ NodeRows node_rows(const int* rowmap, int n, long long nnz, long long n_blocks) {
    NodeRows q{0, 0, 0, false};
    const long long r0 = (long long)rowmap[3 * n] - 1, r1 = (long long)rowmap[3 * n + 1] - 1;
    const long long r2 = (long long)rowmap[3 * n + 2] - 1, r3 = (long long)rowmap[3 * n + 3] - 1;
    const long long len = r1 - r0;
    if (r0 < 0 || len < 3 || (len - 3) % 3 != 0) return q;
    const long long m = (len - 3) / 3;
    if (r2 - r1 != 2 + 3 * m || r3 - r2 != 1 + 3 * m || r3 > nnz) return q;
    const long long off = r0 - 6LL * n;
    if (off < 0 || off % 9 != 0) return q;
    const long long bb = (long long)n + off / 9;
    if (bb + 1 + m > n_blocks) return q;
    q.r0 = r0;
    q.bb = bb;
    q.m = (int)m;
    q.ok = true;
    return q;
}

// Rank of node hi among the upper neighbours of node lo (binary search of row 3*lo), -1 if absent.
__device__ __forceinline__ int neighbour_rank(const int* col, const NodeRows& lo, int hi) {
    int l = 0, r = lo.m - 1;
    const int target = 3 * hi + 1;  // 1-based column of hi's first DOF
    while (l <= r) {
        const int mid = (l + r) >> 1;
        const int c = col[lo.r0 + 3 + 3 * mid];
        if (c == target) return mid;
        if (c < target) l = mid + 1; else r = mid - 1;
    }
    return -1;
}

constexpr int kElemsPerCta = 16;
constexpr int kNaThreads = 8 * kElemsPerCta;

// dN/dxi of node n at Gauss point gp (ModElementHexa8.f90:211-268 at the points of :278-329).
// Local node signs (ModElementHexa8.f90:185-192, 0-based): x + for nodes 1, 2, 5, 6; y + for
// 2, 3, 6, 7; z + for 4..7.  The Gauss points use the same sign pattern.
__device__ __forceinline__ float sgn_x(int i) { return ((i & 3) == 1 || (i & 3) == 2) ? 1.f : -1.f; }
__device__ __forceinline__ float sgn_y(int i) { return (i & 3) >= 2 ? 1.f : -1.f; }
__device__ __forceinline__ float sgn_z(int i) { return i >= 4 ? 1.f : -1.f; }
__device__ __forceinline__ void hexa8_dN(int gp, int n, float d[3]) {
    const float g3 = 0.57735026918962576f;  // 1/sqrt(3), weight 1
    const float x0 = sgn_x(gp) * g3, x1 = sgn_y(gp) * g3, x2 = sgn_z(gp) * g3;
    const float s0 = sgn_x(n), s1 = sgn_y(n), s2 = sgn_z(n);
    d[0] = 0.125f * s0 * (1.f + s1 * x1) * (1.f + s2 * x2);
    d[1] = 0.125f * s1 * (1.f + s0 * x0) * (1.f + s2 * x2);
    d[2] = 0.125f * s2 * (1.f + s0 * x0) * (1.f + s1 * x1);
}

// Compressible Neo-Hookean element loop of 16 elements per CTA: Gauss-point update, internal
// force and the 36 node-pair stiffness blocks of every element, reduced into the block scratch.
// FP32 element arithmetic on element-local coordinate and displacement differences formed in
// FP64; det F and ln J in FP64 (cnh_update).
__global__ void __launch_bounds__(kNaThreads) cnh_noalloc_kernel(int n_nodes, int n_elem, const double* X,
                                                                 const double* U, const int* conn, const int* rowmap,
                                                                 const int* col, long long nnz, long long n_blocks,
                                                                 float mu, float lambda, double* fint, float* blocks,
                                                                 int* bad) {
    __shared__ __align__(16) float s_dx[kElemsPerCta][8][4];        // X_n - X_0 (FP32)
    __shared__ __align__(16) float s_du[kElemsPerCta][8][4];        // u_n - u_0 (FP32)
    __shared__ __align__(16) float s_g[kElemsPerCta][8][8][4];      // [e][gp][node]: grad N (current)
    __shared__ __align__(16) float s_ds[kElemsPerCta][8][28];       // [e][gp]: w D (21), w sigma (6)
    __shared__ int s_node[kElemsPerCta][8];
    __shared__ int s_elem_bad[kElemsPerCta];
    const int t = threadIdx.x, el = t >> 3, j = t & 7;
    const int e = blockIdx.x * kElemsPerCta + el;
    const bool live = e < n_elem;
    if (j == 0) s_elem_bad[el] = live ? 0 : kBadMesh;
    __syncthreads();
    int nid = -1;
    if (live) {
        nid = conn[8 * (size_t)e + j] - 1;
        if (nid < 0 || nid >= n_nodes) {
            atomicOr(&s_elem_bad[el], kBadMesh);
            if (live) atomicOr(bad, kBadMesh);
            nid = -1;
        }
    }
    s_node[el][j] = nid;
    __syncthreads();
    const bool elem_ok = s_elem_bad[el] == 0;
    if (elem_ok) {
        // element-local differences in FP64, then FP32 (sum_n dN_n/dxi = 0 leaves J unchanged)
        const int n0 = s_node[el][0];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s_dx[el][j][d] = (float)(X[3 * (size_t)nid + d] - X[3 * (size_t)n0 + d]);
            s_du[el][j][d] = (float)(U[3 * (size_t)nid + d] - U[3 * (size_t)n0 + d]);
        }
    }
    __syncthreads();
    // ---- Gauss point j of element el ----
    if (elem_ok) {
        const int gp = j;
        float JX[3][3] = {}, Ju[3][3] = {};
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            float dn[3];
            hexa8_dN(gp, n, dn);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    JX[i][k] += dn[i] * s_dx[el][n][k];
                    Ju[i][k] += dn[i] * s_du[el][n][k];
                }
        }
        float Jc[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k) Jc[i][k] = JX[i][k] + Ju[i][k];
        const float dX = ceos::det3(JX), dC = ceos::det3(Jc);
        const bool geom_ok = dX > 1e-13f && dC > 1e-13f;
        float JXi[3][3], Jci[3][3];
        ceos::inv3(JX, geom_ok ? dX : 1.f, JXi);
        ceos::inv3(Jc, geom_ok ? dC : 1.f, Jci);
        float F[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                F[i][k] = (i == k ? 1.f : 0.f) + JXi[k][0] * Ju[0][i] + JXi[k][1] * Ju[1][i] + JXi[k][2] * Ju[2][i];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            float dn[3];
            hexa8_dN(gp, n, dn);
#pragma unroll
            for (int k = 0; k < 3; ++k)
                s_g[el][gp][n][k] = geom_ok ? Jci[k][0] * dn[0] + Jci[k][1] * dn[1] + Jci[k][2] * dn[2] : 0.f;
        }
        float sig[6], D[21];
        if (geom_ok) {
            const float p[2] = {mu, lambda};
            ceos::cnh_update<float>(F, p, sig, D);
        } else {
            atomicOr(bad, kBadGeometry);
        }
        const float w = geom_ok ? dC : 0.f;  // Gauss weight 1 (Hexa8 full integration)
#pragma unroll
        for (int k = 0; k < 21; ++k) s_ds[el][gp][k] = geom_ok ? w * D[k] : 0.f;
#pragma unroll
        for (int k = 0; k < 6; ++k) s_ds[el][gp][21 + k] = geom_ok ? w * sig[k] : 0.f;
    }
    __syncthreads();
    if (!elem_ok) return;
    // ---- node b = j of element el: f_int of b and the blocks (b, b+1..b+npair mod 8) ----
    const int b = j;
    const int npair = (b < 4) ? 4 : 3;
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;
    float Kd[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float Ko[4][9];
#pragma unroll
    for (int o = 0; o < 4; ++o)
#pragma unroll
        for (int k = 0; k < 9; ++k) Ko[o][k] = 0.f;
    for (int gp = 0; gp < 8; ++gp) {
        const float* ds = s_ds[el][gp];
        const float gx = s_g[el][gp][b][0], gy = s_g[el][gp][b][1], gz = s_g[el][gp][b][2];
        const float s0 = ds[21], s1 = ds[22], s2 = ds[23], s3 = ds[24], s4 = ds[25], s5 = ds[26];
        const float q0 = s0 * gx + s3 * gy + s5 * gz;
        const float q1 = s3 * gx + s1 * gy + s4 * gz;
        const float q2 = s5 * gx + s4 * gy + s2 * gz;
        f0 += q0; f1 += q1; f2 += q2;
        float DB[6][3];  // D B_b with D read through its upper triangle
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const float d0 = ds[i <= 0 ? ceos::up21(i, 0) : ceos::up21(0, i)];
            const float d1 = ds[i <= 1 ? ceos::up21(i, 1) : ceos::up21(1, i)];
            const float d2 = ds[i <= 2 ? ceos::up21(i, 2) : ceos::up21(2, i)];
            const float d3 = ds[i <= 3 ? ceos::up21(i, 3) : ceos::up21(3, i)];
            const float d4 = ds[i <= 4 ? ceos::up21(i, 4) : ceos::up21(4, i)];
            const float d5 = ds[i <= 5 ? ceos::up21(i, 5) : ceos::up21(5, i)];
            DB[i][0] = d0 * gx + d3 * gy + d5 * gz;
            DB[i][1] = d1 * gy + d3 * gx + d4 * gz;
            DB[i][2] = d2 * gz + d4 * gy + d5 * gx;
        }
        {
            const float geo = gx * q0 + gy * q1 + gz * q2;
            Kd[0] += gx * DB[0][0] + gy * DB[3][0] + gz * DB[5][0] + geo;
            Kd[1] += gx * DB[0][1] + gy * DB[3][1] + gz * DB[5][1];
            Kd[2] += gx * DB[0][2] + gy * DB[3][2] + gz * DB[5][2];
            Kd[3] += gy * DB[1][1] + gx * DB[3][1] + gz * DB[4][1] + geo;
            Kd[4] += gy * DB[1][2] + gx * DB[3][2] + gz * DB[4][2];
            Kd[5] += gz * DB[2][2] + gy * DB[4][2] + gx * DB[5][2] + geo;
        }
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            if (o < npair) {
                const int an = (b + 1 + o) & 7;
                const float ax = s_g[el][gp][an][0], ay = s_g[el][gp][an][1], az = s_g[el][gp][an][2];
                const float geo = ax * q0 + ay * q1 + az * q2;
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
    // ---- scatter: f_int by FP64 atomics, blocks by 16-byte FP32 vector reductions ----
    const int Bn = s_node[el][b];
    atomicAdd(fint + 3 * (size_t)Bn + 0, (double)f0);
    atomicAdd(fint + 3 * (size_t)Bn + 1, (double)f1);
    atomicAdd(fint + 3 * (size_t)Bn + 2, (double)f2);
    const NodeRows rb = node_rows(rowmap, Bn, nnz, n_blocks);
    if (!rb.ok) {
        atomicOr(bad, kBadMesh);
        return;
    }
    {
        float* blk = blocks + rb.bb * 12;
        red_v4_na(blk + 0, Kd[0], Kd[1], Kd[2], 0.f);
        red_v4_na(blk + 4, 0.f, Kd[3], Kd[4], 0.f);
        red_v4_na(blk + 8, 0.f, 0.f, Kd[5], 0.f);
    }
#pragma unroll
    for (int o = 0; o < 4; ++o) {
        if (o < npair) {
            const int An = s_node[el][(b + 1 + o) & 7];
            if (An == Bn) {  // an element that repeats a node has no such node pair in the pattern
                atomicOr(bad, kBadMesh);
                continue;
            }
            const bool a_low = An < Bn;  // the rows of a node pair belong to the smaller node
            const NodeRows lo = a_low ? node_rows(rowmap, An, nnz, n_blocks) : rb;
            const int r = lo.ok ? neighbour_rank(col, lo, a_low ? Bn : An) : -1;
            if (r < 0) {
                atomicOr(bad, kBadMesh);
                continue;
            }
            float* blk = blocks + (lo.bb + 1 + r) * 12;  // r < lo.m, so the block is below n_blocks
            if (a_low) {  // rows of node a: M[k][:]
                red_v4_na(blk + 0, Ko[o][0], Ko[o][1], Ko[o][2], 0.f);
                red_v4_na(blk + 4, Ko[o][3], Ko[o][4], Ko[o][5], 0.f);
                red_v4_na(blk + 8, Ko[o][6], Ko[o][7], Ko[o][8], 0.f);
            } else {      // rows of node b: M[:][l]
                red_v4_na(blk + 0, Ko[o][0], Ko[o][3], Ko[o][6], 0.f);
                red_v4_na(blk + 4, Ko[o][1], Ko[o][4], Ko[o][7], 0.f);
                red_v4_na(blk + 8, Ko[o][2], Ko[o][5], Ko[o][8], 0.f);
            }
        }
    }
}

// Block scratch -> FP64 CSR values, one warp per node row block.  Rows that fail the layout
// check are left unwritten and flagged.
__global__ void __launch_bounds__(256) blocks_to_csr_noalloc(int n_nodes, const int* rowmap, long long nnz,
                                                             long long n_blocks, const float* blocks, double* K,
                                                             int* bad) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; n < n_nodes; n += warps) {
        const NodeRows q = node_rows(rowmap, n, nnz, n_blocks);
        if (!q.ok) {
            if (lane == 0) atomicOr(bad, kBadMesh);
            continue;
        }
        const int m = q.m;
        const float* blk = blocks + q.bb * 12;
        for (int k = 0; k < 3; ++k) {
            const long long rstart = q.r0 + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
            const int ndg = 3 - k, len = ndg + 3 * m;
            for (int p = lane; p < len; p += 32) {
                int jb, l;
                if (p < ndg) { jb = 0; l = k + p; }
                else { const int pp = p - ndg; jb = 1 + pp / 3; l = pp - 3 * (pp / 3); }
                K[rstart + p] = (double)blk[jb * 12 + 4 * k + l];
            }
        }
    }
}

}  // namespace

extern "C" int ceos_cnh_assemble_noalloc(int n_nodes, int n_elem, const double* X_device, const double* U_device,
                                         const int* conn_device, const int* rowmap_device, const int* col_device,
                                         long long nnz, double mu, double lambda, double* fint_device,
                                         double* kval_device, void* stream) {
    if (n_nodes < 1 || n_elem < 1 || !X_device || !U_device || !conn_device || !rowmap_device || !col_device ||
        !fint_device || !kval_device || nnz < 6LL * n_nodes)
        return CEOS_E_ARG;
    // node-pair blocks: one diagonal block per node plus one per upper neighbour
    const long long n_blocks = (long long)n_nodes + (nnz - 6LL * n_nodes) / 9;
    // blocks plus one flag word must fit the 8 MiB static scratch; larger meshes are refused
    if (n_blocks > kAsmScratchBlocks || n_blocks * 48 + 16 > (long long)kAsmScratchBytes) return CEOS_E_ARG;
    float* scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The scratch keeps the previous call's contents: clear the part this call uses.  The flag
    // word after the blocks collects geometry / pattern failures of this call.
    int* bad = reinterpret_cast<int*>(scratch + n_blocks * 12);
    if (cudaMemsetAsync(scratch, 0, (size_t)n_blocks * 48 + 16, s) != cudaSuccess) return CEOS_E_CUDA;
    if (cudaMemsetAsync(fint_device, 0, sizeof(double) * 3 * (size_t)n_nodes, s) != cudaSuccess) return CEOS_E_CUDA;
    const unsigned grid = (unsigned)((n_elem + kElemsPerCta - 1) / kElemsPerCta);
    cnh_noalloc_kernel<<<grid, kNaThreads, 0, s>>>(n_nodes, n_elem, X_device, U_device, conn_device, rowmap_device,
                                                  col_device, nnz, n_blocks, (float)mu, (float)lambda, fint_device,
                                                  scratch, bad);
    if (cudaGetLastError() != cudaSuccess) return CEOS_E_CUDA;
    blocks_to_csr_noalloc<<<(n_nodes + 7) / 8, 256, 0, s>>>(n_nodes, rowmap_device, nnz, n_blocks, scratch,
                                                            kval_device, bad);
    if (cudaGetLastError() != cudaSuccess) return CEOS_E_CUDA;
    int hbad = 0;
    if (cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CEOS_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CEOS_E_CUDA;
    if (hbad & kBadMesh) return CEOS_E_MESH;   // the mesh or pattern does not match (K incomplete)
    if (hbad & kBadGeometry) return 1;         // det J <= 1e-13 in some element (ClassStatus error 1)
    return 0;
}
