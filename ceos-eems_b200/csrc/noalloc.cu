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

__device__ __forceinline__ void red_v4_na(float* p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

// First block of node n in the block layout: n + (number of upper neighbours of nodes < n).
// With the 1-based upper CSR of the reference, row 3n starts at rowmap[3n]-1 = 6n + 9*(that sum).
__device__ __forceinline__ long long first_block(const int* rowmap, int n) {
    const long long rs = (long long)rowmap[3 * n] - 1;
    return (long long)n + (rs - 6LL * n) / 9;
}

// Rank of node hi among the upper neighbours of node lo, read from row 3*lo of the CSR.
__device__ __forceinline__ int neighbour_rank(const int* rowmap, const int* col, int lo, int hi) {
    const long long rs = (long long)rowmap[3 * lo] - 1;
    const int m = (rowmap[3 * lo + 1] - rowmap[3 * lo] - 3) / 3;
    int l = 0, r = m - 1;
    const int target = 3 * hi + 1;  // 1-based column of hi's first DOF
    while (l <= r) {
        const int mid = (l + r) >> 1;
        const int c = col[rs + 3 + 3 * mid];
        if (c == target) return mid;
        if (c < target) l = mid + 1; else r = mid - 1;
    }
    return -1;
}

// One thread per element: Gauss-point update (compressible Neo-Hookean), internal force and
// the 36 node-pair stiffness blocks, reduced into the block scratch.  FP32 element arithmetic.
__global__ void __launch_bounds__(128) cnh_noalloc_kernel(int n_elem, const double* X, const double* U,
                                                          const int* conn, const int* rowmap, const int* col,
                                                          float mu, float lambda, double* fint, float* blocks,
                                                          int* bad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    int nd[8];
    float Xe[8][3], Ue[8][3];
    for (int a = 0; a < 8; ++a) {
        nd[a] = conn[8 * e + a] - 1;
        for (int d = 0; d < 3; ++d) {
            Xe[a][d] = (float)X[3 * nd[a] + d];
            Ue[a][d] = (float)U[3 * nd[a] + d];
        }
    }
    const float g3 = 0.57735026918962576f;  // 1/sqrt(3): 2x2x2 Gauss points, weight 1
    float fe[8][3] = {};
    float Kb[36][9] = {};  // pair (a <= b) in row-major upper order, block rows = node a
    // Hexa8 node signs (ModElementHexa8.f90:185-192): x + for local nodes 1,2,5,6; y + for 2,3,6,7;
    // z + for 4..7 (0-based)
    auto sx = [](int i) { return ((i & 3) == 1 || (i & 3) == 2) ? 1.f : -1.f; };
    auto sy = [](int i) { return (i & 3) >= 2 ? 1.f : -1.f; };
    auto sz = [](int i) { return i >= 4 ? 1.f : -1.f; };
    for (int gp = 0; gp < 8; ++gp) {
        const float xi[3] = {sx(gp) * g3, sy(gp) * g3, sz(gp) * g3};
        float dN[8][3];
        for (int i = 0; i < 8; ++i) {
            const float s0 = sx(i), s1 = sy(i), s2 = sz(i);
            dN[i][0] = s0 * (1.f + s1 * xi[1]) * (1.f + s2 * xi[2]) * 0.125f;
            dN[i][1] = s1 * (1.f + s0 * xi[0]) * (1.f + s2 * xi[2]) * 0.125f;
            dN[i][2] = s2 * (1.f + s0 * xi[0]) * (1.f + s1 * xi[1]) * 0.125f;
        }
        float JX[3][3] = {}, Jc[3][3] = {};
        for (int n = 0; n < 8; ++n)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    JX[i][j] += dN[n][i] * Xe[n][j];
                    Jc[i][j] += dN[n][i] * (Xe[n][j] + Ue[n][j]);
                }
        const float dX = ceos::det3(JX), dC = ceos::det3(Jc);
        if (!(dX > 1e-13f) || !(dC > 1e-13f)) {
            atomicOr(bad, 1);
            continue;
        }
        float JXi[3][3], Jci[3][3];
        ceos::inv3(JX, dX, JXi);
        ceos::inv3(Jc, dC, Jci);
        float F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        float g[8][3];
        for (int n = 0; n < 8; ++n) {
            float gX[3];
            for (int j = 0; j < 3; ++j) {
                gX[j] = JXi[j][0] * dN[n][0] + JXi[j][1] * dN[n][1] + JXi[j][2] * dN[n][2];
                g[n][j] = Jci[j][0] * dN[n][0] + Jci[j][1] * dN[n][1] + Jci[j][2] * dN[n][2];
            }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) F[i][j] += Ue[n][i] * gX[j];
        }
        const float p[2] = {mu, lambda};
        float sig[6], D[21];
        ceos::cnh_update<float>(F, p, sig, D);
        for (int k = 0; k < 6; ++k) sig[k] *= dC;
        for (int k = 0; k < 21; ++k) D[k] *= dC;
        auto Dij = [&](int i, int j) { return i <= j ? D[ceos::up21(i, j)] : D[ceos::up21(j, i)]; };
        float q[8][3], DB[8][6][3];
        for (int b = 0; b < 8; ++b) {
            const float gx = g[b][0], gy = g[b][1], gz = g[b][2];
            q[b][0] = sig[0] * gx + sig[3] * gy + sig[5] * gz;
            q[b][1] = sig[3] * gx + sig[1] * gy + sig[4] * gz;
            q[b][2] = sig[5] * gx + sig[4] * gy + sig[2] * gz;
            for (int d = 0; d < 3; ++d) fe[b][d] += q[b][d];
            for (int i = 0; i < 6; ++i) {
                DB[b][i][0] = Dij(i, 0) * gx + Dij(i, 3) * gy + Dij(i, 5) * gz;
                DB[b][i][1] = Dij(i, 1) * gy + Dij(i, 3) * gx + Dij(i, 4) * gz;
                DB[b][i][2] = Dij(i, 2) * gz + Dij(i, 4) * gy + Dij(i, 5) * gx;
            }
        }
        int pidx = 0;
        for (int a = 0; a < 8; ++a)
            for (int b = a; b < 8; ++b, ++pidx) {
                const float ax = g[a][0], ay = g[a][1], az = g[a][2];
                const float geo = ax * q[b][0] + ay * q[b][1] + az * q[b][2];
                for (int l = 0; l < 3; ++l) {
                    Kb[pidx][0 * 3 + l] += ax * DB[b][0][l] + ay * DB[b][3][l] + az * DB[b][5][l];
                    Kb[pidx][1 * 3 + l] += ay * DB[b][1][l] + ax * DB[b][3][l] + az * DB[b][4][l];
                    Kb[pidx][2 * 3 + l] += az * DB[b][2][l] + ay * DB[b][4][l] + ax * DB[b][5][l];
                }
                Kb[pidx][0] += geo; Kb[pidx][4] += geo; Kb[pidx][8] += geo;
            }
    }
    for (int a = 0; a < 8; ++a)
        for (int d = 0; d < 3; ++d) atomicAdd(fint + 3 * (size_t)nd[a] + d, (double)fe[a][d]);
    int pidx = 0;
    for (int a = 0; a < 8; ++a)
        for (int b = a; b < 8; ++b, ++pidx) {
            const float* M = Kb[pidx];  // rows of node a, columns of node b
            if (a == b) {
                float* blk = blocks + first_block(rowmap, nd[a]) * 12;
                red_v4_na(blk + 0, M[0], M[1], M[2], 0.f);
                red_v4_na(blk + 4, 0.f, M[4], M[5], 0.f);
                red_v4_na(blk + 8, 0.f, 0.f, M[8], 0.f);
                continue;
            }
            const bool a_low = nd[a] < nd[b];
            const int lo = a_low ? nd[a] : nd[b], hi = a_low ? nd[b] : nd[a];
            const int r = neighbour_rank(rowmap, col, lo, hi);
            if (r < 0) { atomicOr(bad, 2); continue; }
            float* blk = blocks + (first_block(rowmap, lo) + 1 + r) * 12;
            if (a_low) {
                red_v4_na(blk + 0, M[0], M[1], M[2], 0.f);
                red_v4_na(blk + 4, M[3], M[4], M[5], 0.f);
                red_v4_na(blk + 8, M[6], M[7], M[8], 0.f);
            } else {
                red_v4_na(blk + 0, M[0], M[3], M[6], 0.f);
                red_v4_na(blk + 4, M[1], M[4], M[7], 0.f);
                red_v4_na(blk + 8, M[2], M[5], M[8], 0.f);
            }
        }
}

// Block scratch -> FP64 CSR values, one warp per node row block.
__global__ void __launch_bounds__(256) blocks_to_csr_noalloc(int n_nodes, const int* rowmap, const float* blocks,
                                                             double* K) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; n < n_nodes; n += warps) {
        const long long rs = (long long)rowmap[3 * n] - 1;
        const int m = (rowmap[3 * n + 1] - rowmap[3 * n] - 3) / 3;
        const float* blk = blocks + first_block(rowmap, n) * 12;
        for (int k = 0; k < 3; ++k) {
            const long long rstart = rs + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
            const int ndg = 3 - k, len = ndg + 3 * m;
            for (int p = lane; p < len; p += 32) {
                int j, l;
                if (p < ndg) { j = 0; l = k + p; }
                else { const int pp = p - ndg; j = 1 + pp / 3; l = pp - 3 * (pp / 3); }
                K[rstart + p] = (double)blk[j * 12 + 4 * k + l];
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
    cnh_noalloc_kernel<<<(n_elem + 127) / 128, 128, 0, s>>>(n_elem, X_device, U_device, conn_device, rowmap_device,
                                                            col_device, (float)mu, (float)lambda, fint_device,
                                                            scratch, bad);
    if (cudaGetLastError() != cudaSuccess) return CEOS_E_CUDA;
    blocks_to_csr_noalloc<<<(n_nodes + 7) / 8, 256, 0, s>>>(n_nodes, rowmap_device, scratch, kval_device);
    if (cudaGetLastError() != cudaSuccess) return CEOS_E_CUDA;
    int hbad = 0;
    if (cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CEOS_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CEOS_E_CUDA;
    if (hbad & 1) return 1;  // det J <= 1e-13 in some element (ClassStatus error 1)
    if (hbad & 2) return CEOS_E_MESH;
    return 0;
}
