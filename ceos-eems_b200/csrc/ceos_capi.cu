// ceos_capi.cu -- the C ABI (include/ceos_gpu.h): handle, CSR pattern, slot map, launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ceos_gpu.h"
#include "ceos_handle.h"
#include "element_kernel.cuh"
#include "schedule.h"

namespace ceos {


namespace {

// dN table with the arithmetic of GetDifShapeFunctions_Hexa8 (ModElementHexa8.f90:211-268)
// at the points of AllocateGaussPointsParameters_Hexa8 (:278-329).
void hexa8_dN_table(double out[8][8][3]) {
    const double x = 1.0 / std::sqrt(3.0);
    for (int gp = 0; gp < 8; ++gp) {
        const double xi = kSign[gp][0] * x, eta = kSign[gp][1] * x, zeta = kSign[gp][2] * x;
        for (int i = 0; i < 8; ++i) {
            out[gp][i][0] = kSign[i][0] * (1.0 + kSign[i][1] * eta) * (1.0 + kSign[i][2] * zeta) / 8.0;
            out[gp][i][1] = kSign[i][1] * (1.0 + kSign[i][0] * xi) * (1.0 + kSign[i][2] * zeta) / 8.0;
            out[gp][i][2] = kSign[i][2] * (1.0 + kSign[i][0] * xi) * (1.0 + kSign[i][1] * eta) / 8.0;
        }
    }
}

int model_nparams(int model) {
    switch (model) {
        case M_CNH: return ModelInfo<M_CNH>::nparams;
        case M_NH_Q1P0: return ModelInfo<M_NH_Q1P0>::nparams;
        case M_SVK: return ModelInfo<M_SVK>::nparams;
        case M_J2_SMALL: return ModelInfo<M_J2_SMALL>::nparams;
        case M_VISCO_PRONY: return ModelInfo<M_VISCO_PRONY>::nparams;
        case M_J2_FINITE: return ModelInfo<M_J2_FINITE>::nparams;
        case M_VISCO_VAR: return ModelInfo<M_VISCO_VAR>::nparams;
        case M_EXTERNAL: return ModelInfo<M_EXTERNAL>::nparams;
    }
    return -1;
}
int model_nstate(int model) {
    switch (model) {
        case M_CNH: return 0;
        case M_NH_Q1P0: return 0;
        case M_SVK: return 0;
        case M_J2_SMALL: return ModelInfo<M_J2_SMALL>::nstate;
        case M_VISCO_PRONY: return ModelInfo<M_VISCO_PRONY>::nstate;
        case M_J2_FINITE: return ModelInfo<M_J2_FINITE>::nstate;
        case M_VISCO_VAR: return ModelInfo<M_VISCO_VAR>::nstate;
        case M_EXTERNAL: return ModelInfo<M_EXTERNAL>::nstate;
    }
    return -1;
}
void model_init_state(int model, double* st) {
    const int ns = model_nstate(model);
    for (int i = 0; i < ns; ++i) st[i] = 0.0;
    if (model == M_J2_FINITE) st[0] = st[1] = st[2] = 1.0;  // Cp^{-1} = I
    if (model == M_VISCO_VAR) st[0] = st[4] = st[8] = 1.0;  // Fv = I (ModViscoelasticMatrix.f90:124-131)
}

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t err_ = (call);                                            \
        if (err_ != cudaSuccess) {                                            \
            h->msg = std::string(#call) + ": " + cudaGetErrorString(err_);   \
            return CEOS_E_CUDA;                                               \
        }                                                                     \
    } while (0)

template <typename T>
size_t elem_smem(const Handle* h) { return SmemLayout<T>(h->ns_used, h->param_mode == 1 ? h->n_params : 0).total; }

// Streams and events of the banded assembly, created at its first evaluation.
int ensure_band_streams(Handle* h) {
    if (h->band_stream) return 0;
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithFlags(&h->band_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithPriority(&h->conv_stream, cudaStreamNonBlocking, hi));  // hi: the greatest priority
    CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    h->ev_band.assign(h->n_bands, nullptr);
    h->ev_bconv.assign(h->n_bands, nullptr);
    for (auto& ev : h->ev_band) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (auto& ev : h->ev_bconv) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return 0;
}

// The launches of one evaluation range.  CEOS_MIXED with a tangent, two-pass assembly (default):
// the element loop over elements [e0, e1) reducing FP32 node-pair blocks into the scratch, then
// the conversion of the items of element slab `slab` (every item for slab -1).  Fused assembly:
// one launch over the queue items of slab `slab` (the whole queue for slab -1).  Otherwise: the
// element loop over [e0, e1) with the static tile schedule (K by FP64 atomics in CEOS_FP64 mode,
// no K without a tangent).
template <typename T, int MODEL>
int launch_model(Handle* h, double dt, const double* dU, double* dfint, double* dkval, cudaStream_t s, int e0, int e1,
                 int slab) {
    ElemArgs<T> a{};
    a.n_elem = h->n_elem;
    for (int k = 0; k < 12; ++k) a.pu[k] = T(0);
    if (h->param_mode == 0)
        for (int k = 0; k < h->n_params && k < 12; ++k) a.pu[k] = (T)h->host_params[k];
    for (int k = 0; k < 4; ++k) a.ebr[k] = T(0);
    if (MODEL == M_VISCO_PRONY && h->param_mode == 0)
        for (int k = 0; k < 4 && k < (int)h->host_params[2]; ++k)
            a.ebr[k] = (T)std::exp(-dt / (2.0 * h->host_params[4 + 2 * k]));
    a.X = h->d_X;
    a.jxi = h->d_jxi;
    a.U = dU;
    a.conn = h->d_conn;
    a.nup = h->d_nup;
    a.ranks = h->d_ranks;
    a.fint = dfint;
    a.kval = dkval;
    a.st_old = reinterpret_cast<const T*>(h->d_state[h->cur_old]);
    a.st_new = reinterpret_cast<T*>(h->d_state[1 - h->cur_old]);
    a.ld = h->ld;
    a.ns_used = h->ns_used;
    a.n_pe = h->param_mode == 1 ? h->n_params : 0;
    a.params = reinterpret_cast<const T*>(h->d_params);
    a.param_mode = h->param_mode;
    a.n_params = h->n_params;
    a.mat_id = h->d_mat_id;
    a.dt = dt;
    a.elem_status = h->d_elem_status;
    a.status_count = h->d_status_count;
    a.gp_stress = (h->options & CEOS_OPT_STORE_STRESS) ? reinterpret_cast<T*>(h->d_gp_stress) : nullptr;
    const size_t smem = elem_smem<T>(h);
    const bool timed = (h->options & CEOS_OPT_TIME_KERNELS) && h->ev_k0;
    if constexpr (sizeof(T) == 4) {
        if (dkval && h->assembly == CEOS_ASSEMBLY_BANDED) {
            // the whole mesh band by band (every band is a slab of its own; `slab` is not used):
            // even element bands on s, odd ones on band_stream, conversions on conv_stream
            a.rs = h->d_blk0;
            a.kblk = h->d_kblk;
            a.ring_mask = h->band_ring - 1;
            a.csr_rs = h->d_rs;
            a.conv_meta = static_cast<const longlong2*>(h->d_bconv_meta);  // the bands' conversion items
            a.sched_err = h->d_sched_err;
            {
                const int r = ensure_band_streams(h);
                if (r) return r;
            }
            CK(cudaFuncSetAttribute(element_loop_kernel<float, MODEL, SCATTER_RING>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            if (timed) CK(cudaEventRecord(h->ev_k0, s));
            CK(cudaEventRecord(h->ev_fork, s));
            CK(cudaStreamWaitEvent(h->band_stream, h->ev_fork, 0));
            CK(cudaStreamWaitEvent(h->conv_stream, h->ev_fork, 0));
            if (h->copy_f) CK(cudaStreamWaitEvent(h->copy_stream, h->ev_fork, 0));
            int n_done = 0;
            for (int c = 0; c < h->n_bands; ++c) {
                cudaStream_t st = (c & 1) ? h->band_stream : s;
                // ring slots: every row below band_node_end[c - depth] is converted and zeroed
                if (c >= h->band_depth) CK(cudaStreamWaitEvent(st, h->ev_bconv[c - h->band_depth], 0));
                a.e_begin = h->band_e[c];
                a.e_end = h->band_e[c + 1];
                const int n_tiles = (a.e_end - a.e_begin + kTileE - 1) / kTileE;
                element_loop_kernel<float, MODEL, SCATTER_RING><<<std::min(n_tiles, h->grid_cap), kThreads, smem, st>>>(a);
                CK(cudaGetLastError());
                CK(cudaEventRecord(h->ev_band[c], st));
                // rows of band c: every band <= c has reduced (band c - 1 was waited for before the
                // conversion of band c - 1, earlier in conv_stream)
                CK(cudaStreamWaitEvent(h->conv_stream, h->ev_band[c], 0));
                const int j0 = h->band_conv[c], j1 = h->band_conv[c + 1];
                if (j1 > j0) {
                    csr_convert_kernel<<<std::min(j1 - j0, h->conv_grid), kThreads, kBulkSmem, h->conv_stream>>>(
                        a, nullptr, j0, j1);
                    CK(cudaGetLastError());
                }
                CK(cudaEventRecord(h->ev_bconv[c], h->conv_stream));
                const int n_end = h->band_node_end[c];
                if (h->copy_f && n_end > n_done) {  // host-buffer call: the finished rows go to the host now
                    CK(cudaStreamWaitEvent(h->copy_stream, h->ev_bconv[c], 0));
                    CK(cudaMemcpyAsync(h->copy_f + 3 * (size_t)n_done, dfint + 3 * (size_t)n_done,
                                       3 * (size_t)(n_end - n_done) * sizeof(double), cudaMemcpyDeviceToHost,
                                       h->copy_stream));
                    const long long k0 = h->rs[n_done], k1 = n_end < h->n_nodes ? h->rs[n_end] : h->nnz;
                    CK(cudaMemcpyAsync(h->copy_k + k0, dkval + k0, (size_t)(k1 - k0) * sizeof(double),
                                       cudaMemcpyDeviceToHost, h->copy_stream));
                }
                n_done = n_end;
            }
            CK(cudaStreamWaitEvent(s, h->ev_bconv[h->n_bands - 1], 0));  // joins every band and conversion
            if (timed) {
                CK(cudaEventRecord(h->ev_k1, s));
                CK(cudaEventRecord(h->ev_k2, s));
            }
            return 0;
        }
        if (dkval && h->assembly == CEOS_ASSEMBLY_TWO_PASS) {
            a.e_begin = e0;
            a.e_end = e1;
            a.rs = h->d_blk0;
            a.kblk = h->d_kblk;
            a.ring_mask = h->scratch_mask;  // covers every block: no slot is shared
            a.csr_rs = h->d_rs;
            a.conv_meta = static_cast<const longlong2*>(h->d_conv_meta);  // the two-pass conversion items
            a.sched_err = h->d_sched_err;
            const int j0 = slab < 0 ? 0 : h->slab_conv[slab], j1 = slab < 0 ? h->n_conv2 : h->slab_conv[slab + 1];
            CK(cudaFuncSetAttribute(element_loop_kernel<float, MODEL, SCATTER_RING>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const int n_tiles = (e1 - e0 + kTileE - 1) / kTileE;
            if (timed) CK(cudaEventRecord(h->ev_k0, s));
            if (n_tiles > 0) {
                element_loop_kernel<float, MODEL, SCATTER_RING><<<std::min(n_tiles, h->grid_cap), kThreads, smem, s>>>(a);
                CK(cudaGetLastError());
            }
            if (timed) CK(cudaEventRecord(h->ev_k1, s));
            if (j1 > j0) {
                csr_convert_kernel<<<std::min(j1 - j0, h->conv_grid), kThreads, kBulkSmem, s>>>(a, h->d_conv_order,
                                                                                                 j0, j1);
                CK(cudaGetLastError());
            }
            if (timed) CK(cudaEventRecord(h->ev_k2, s));
            return 0;
        }
        if (dkval) {
            a.e_begin = 0;
            a.e_end = h->n_elem;
            a.rs = h->d_blk0;
            a.kblk = h->d_kblk;
            a.ring_mask = h->ring_blocks - 1;
            a.csr_rs = h->d_rs;
            a.queue = h->d_queue;
            a.q_begin = slab < 0 ? 0 : h->slab_q[slab];                 // slab -1: the whole queue
            a.q_end = slab < 0 ? (int)h->queue.size() : h->slab_q[slab + 1];
            a.ticket = h->d_ticket;
            a.tile_done = h->d_flags;
            a.conv_done = h->d_flags + h->n_tiles;
            a.epoch = h->epoch;
            a.conv = static_cast<const int4*>(h->d_conv);
            a.tile_wait = static_cast<const int2*>(h->d_tile_wait);
            a.sched_err = h->d_sched_err;
            CK(cudaMemsetAsync(h->d_ticket, 0, sizeof(unsigned), s));
            CK(cudaFuncSetAttribute(element_assemble_kernel<MODEL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const int nq = a.q_end - a.q_begin;
            if (timed) CK(cudaEventRecord(h->ev_k0, s));
            if (nq > 0) {
                element_assemble_kernel<MODEL><<<std::min(nq, h->grid_cap), kThreads, smem, s>>>(a);
                CK(cudaGetLastError());
            }
            if (timed) {
                CK(cudaEventRecord(h->ev_k1, s));
                CK(cudaEventRecord(h->ev_k2, s));
            }
            return 0;
        }
    }
    a.e_begin = e0;
    a.e_end = e1;
    a.rs = h->d_rs;
    CK(cudaFuncSetAttribute(element_loop_kernel<T, MODEL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int n_tiles = (a.e_end - a.e_begin + kTileE - 1) / kTileE;
    const int grid = std::min(n_tiles, h->grid_cap);
    if (timed) CK(cudaEventRecord(h->ev_k0, s));
    if (n_tiles > 0) {
        element_loop_kernel<T, MODEL><<<grid, kThreads, smem, s>>>(a);
        CK(cudaGetLastError());
    }
    if (timed) {
        CK(cudaEventRecord(h->ev_k1, s));
        CK(cudaEventRecord(h->ev_k2, s));
    }
    return 0;
}

template <typename T>
int launch_elem(Handle* h, double dt, const double* dU, double* dfint, double* dkval, cudaStream_t s, int e0, int e1,
                int slab) {
    switch (h->model) {
        case M_CNH: return launch_model<T, M_CNH>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_NH_Q1P0: return launch_model<T, M_NH_Q1P0>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_SVK: return launch_model<T, M_SVK>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_J2_SMALL: return launch_model<T, M_J2_SMALL>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_VISCO_PRONY: return launch_model<T, M_VISCO_PRONY>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_J2_FINITE: return launch_model<T, M_J2_FINITE>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_VISCO_VAR: return launch_model<T, M_VISCO_VAR>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
        case M_EXTERNAL: return launch_model<T, M_EXTERNAL>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
    }
    return CEOS_E_MODEL;
}

template <typename K>
int blocks_per_sm(K kernel, size_t smem) {
    int per_sm = 1;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
    return (e != cudaSuccess || per_sm < 1) ? 1 : per_sm;
}

// Resident CTAs per SM of the evaluation kernels of this handle (in mixed mode the fewer of the
// two-pass element kernel and the fused kernel, which share one shared-memory layout).
template <typename T, int MODEL>
int model_blocks_per_sm(Handle* h) {
    const size_t smem = elem_smem<T>(h);
    if constexpr (sizeof(T) == 4)
        return std::min(blocks_per_sm(element_assemble_kernel<MODEL>, smem),
                        blocks_per_sm(element_loop_kernel<float, MODEL, SCATTER_RING>, smem));
    return blocks_per_sm(element_loop_kernel<T, MODEL>, smem);
}

template <typename T>
int occupancy_grid(Handle* h) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    int per_sm = 1;
    switch (h->model) {
        case M_CNH: per_sm = model_blocks_per_sm<T, M_CNH>(h); break;
        case M_NH_Q1P0: per_sm = model_blocks_per_sm<T, M_NH_Q1P0>(h); break;
        case M_SVK: per_sm = model_blocks_per_sm<T, M_SVK>(h); break;
        case M_J2_SMALL: per_sm = model_blocks_per_sm<T, M_J2_SMALL>(h); break;
        case M_VISCO_PRONY: per_sm = model_blocks_per_sm<T, M_VISCO_PRONY>(h); break;
        case M_J2_FINITE: per_sm = model_blocks_per_sm<T, M_J2_FINITE>(h); break;
        case M_VISCO_VAR: per_sm = model_blocks_per_sm<T, M_VISCO_VAR>(h); break;
        case M_EXTERNAL: per_sm = model_blocks_per_sm<T, M_EXTERNAL>(h); break;
    }
    h->blocks_per_sm = per_sm;
    return sms * per_sm;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// CSR pattern of AllocateKgSparseUpperTriangular (ModFEMAnalysis.f90:209-273): row 3n+k holds,
// in increasing order, the columns 3n+k..3n+2 of its own node and the three DOFs of every
// neighbour node with a larger id.  Built from sorted node adjacency lists, which gives the
// same sorted distinct columns as the reference's per-row linked lists
// (ModSparseVectorRoutines.f90:222-312) filtered to col >= row
// (ModSparseMatrixRoutines.f90:573-609).
// ---------------------------------------------------------------------------------------
int build_pattern(Handle* h, const int* conn1) {
    const int N = h->n_nodes, E = h->n_elem;
    std::vector<int> deg(N + 1, 0);
    // upper neighbours of each node: count candidate pairs, then sort + unique
    std::vector<long long> cnt(N + 1, 0);
    for (int e = 0; e < E; ++e)
        for (int i = 0; i < 8; ++i) {
            const int a = conn1[8 * e + i] - 1;
            for (int j = 0; j < 8; ++j) {
                const int b = conn1[8 * e + j] - 1;
                if (b > a) cnt[a + 1]++;
            }
        }
    for (int n = 0; n < N; ++n) cnt[n + 1] += cnt[n];
    std::vector<int> buf(cnt[N]);
    std::vector<long long> fill(cnt.begin(), cnt.end() - 1);
    std::vector<char> used(N, 0);
    for (int e = 0; e < E; ++e)
        for (int i = 0; i < 8; ++i) {
            const int a = conn1[8 * e + i] - 1;
            used[a] = 1;
            for (int j = 0; j < 8; ++j) {
                const int b = conn1[8 * e + j] - 1;
                if (b > a) buf[fill[a]++] = b;
            }
        }
    for (int n = 0; n < N; ++n)
        if (!used[n]) {
            h->msg = "node " + std::to_string(n + 1) + " belongs to no element";
            return CEOS_E_MESH;
        }
    h->up_ptr.assign(N + 1, 0);
    h->up_list.clear();
    h->up_list.reserve(cnt[N] / 4 + 16);
    for (int n = 0; n < N; ++n) {
        auto b0 = buf.begin() + cnt[n], b1 = buf.begin() + cnt[n + 1];
        std::sort(b0, b1);
        auto last = std::unique(b0, b1);
        h->up_list.insert(h->up_list.end(), b0, last);
        h->up_ptr[n + 1] = (long long)h->up_list.size();
    }
    // node row starts: row 3n has 3 + 3m entries, row 3n+1 2 + 3m, row 3n+2 1 + 3m
    h->rs.assign(N, 0);
    h->nup.assign(N, 0);
    long long pos = 0;
    for (int n = 0; n < N; ++n) {
        const int m = (int)(h->up_ptr[n + 1] - h->up_ptr[n]);
        h->rs[n] = pos;
        h->nup[n] = m;
        pos += 6 + 9LL * m;
        if (m > 255) {
            h->msg = "node with more than 255 neighbours";
            return CEOS_E_MESH;
        }
    }
    h->nnz = pos;
    // per element: rank of the larger node among the smaller node's upper neighbours
    h->ranks.assign((size_t)E * 32, 0);
    for (int e = 0; e < E; ++e)
        for (int i = 0; i < 8; ++i)
            for (int j = i + 1; j < 8; ++j) {
                const int A = conn1[8 * e + i] - 1, B = conn1[8 * e + j] - 1;
                if (A == B) {
                    h->msg = "element " + std::to_string(e + 1) + " repeats a node";
                    return CEOS_E_MESH;
                }
                const int lo = std::min(A, B), hi = std::max(A, B);
                const int* b0 = h->up_list.data() + h->up_ptr[lo];
                const int* b1 = h->up_list.data() + h->up_ptr[lo + 1];
                const int r = (int)(std::lower_bound(b0, b1, hi) - b0);
                h->ranks[(size_t)e * 32 + pair_index(i, j)] = (uint8_t)r;
            }
    return 0;
}

}  // namespace ceos

namespace ceos {
static void plan_slab_bounds(Handle* h);
static int build_schedule(Handle* h);
}  // namespace ceos

using namespace ceos;

extern "C" int ceos_create(const ceos_mesh* mesh, const ceos_material* mats, int n_mat, int precision_mode,
                           int device, void** handle) {
    if (!mesh || !mats || n_mat < 1 || !handle || mesh->n_nodes < 1 || mesh->n_elem < 1 || !mesh->X || !mesh->conn)
        return CEOS_E_ARG;
    if (precision_mode != CEOS_FP64 && precision_mode != CEOS_MIXED) return CEOS_E_ARG;
    Handle* h = new Handle();
    *handle = nullptr;
    h->n_nodes = mesh->n_nodes;
    h->n_elem = mesh->n_elem;
    h->precision = precision_mode;
    h->device = device;
    h->model = mats[0].model;
    for (int k = 0; k < n_mat; ++k)
        if (mats[k].model != h->model) { delete h; return CEOS_E_MODEL; }
    h->n_params = model_nparams(h->model);
    h->nstate = model_nstate(h->model);
    if (h->n_params < 0) { delete h; return CEOS_E_MODEL; }
    for (int k = 0; k < n_mat; ++k)
        if (mats[k].n_params < h->n_params || !mats[k].params) { delete h; return CEOS_E_ARG; }
    for (long long i = 0; i < 8LL * mesh->n_elem; ++i)
        if (mesh->conn[i] < 1 || mesh->conn[i] > mesh->n_nodes) { delete h; return CEOS_E_MESH; }
    int rc = build_pattern(h, mesh->conn);
    if (rc) { std::fprintf(stderr, "ceos_create: %s\n", h->msg.c_str()); delete h; return rc; }
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) { delete h; return CEOS_E_CUDA; }
    rc = h->allocate_device(mesh, mats, n_mat);
    if (rc) { std::fprintf(stderr, "ceos_create: %s\n", h->msg.c_str()); delete h; return rc; }
    h->grid_cap = (precision_mode == CEOS_FP64) ? occupancy_grid<double>(h) : occupancy_grid<float>(h);
    plan_slab_bounds(h);
    if (precision_mode == CEOS_MIXED) {
        rc = build_schedule(h);
        if (rc) { std::fprintf(stderr, "ceos_create: %s\n", h->msg.c_str()); delete h; return rc; }
    }
    {
        double tab[8][8][3];
        hexa8_dN_table(tab);
        float tabf[8][8][3];
        for (int g = 0; g < 8; ++g)
            for (int n = 0; n < 8; ++n)
                for (int i = 0; i < 3; ++i) tabf[g][n][i] = (float)tab[g][n][i];
        if (cudaMemcpyToSymbol(c_dN, tab, sizeof(tab)) != cudaSuccess ||
            cudaMemcpyToSymbol(c_dNf, tabf, sizeof(tabf)) != cudaSuccess) {
            delete h;
            return CEOS_E_CUDA;
        }
    }
    *handle = h;
    return 0;
}

extern "C" int ceos_pattern(void* handle, int* n_dof, long long* nnz, int* rowmap, int* col, int* row) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    const int N = h->n_nodes;
    if (n_dof) *n_dof = 3 * N;
    if (nnz) *nnz = h->nnz;
    if (h->nnz > 2147483646LL && (rowmap || col || row)) return CEOS_E_ARG;  // 1-based int32 export
    long long k = 0;
    for (int n = 0; n < N; ++n) {
        const long long b0 = h->up_ptr[n], b1 = h->up_ptr[n + 1];
        for (int r = 0; r < 3; ++r) {
            const int irow = 3 * n + r + 1;
            if (rowmap) rowmap[irow - 1] = (int)(k + 1);
            for (int c = r; c < 3; ++c) {
                if (col) col[k] = 3 * n + c + 1;
                if (row) row[k] = irow;
                ++k;
            }
            for (long long q = b0; q < b1; ++q)
                for (int c = 0; c < 3; ++c) {
                    if (col) col[k] = 3 * h->up_list[q] + c + 1;
                    if (row) row[k] = irow;
                    ++k;
                }
        }
    }
    if (rowmap) rowmap[3 * N] = (int)(h->nnz + 1);
    return 0;
}

extern "C" int ceos_slot_map(void* handle, long long* out) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !out) return CEOS_E_ARG;
    // The same arithmetic the kernel uses (element_kernel.cuh, phase B scatter).
    for (int e = 0; e < h->n_elem; ++e) {
        long long* o = out + (size_t)e * 576;
        for (int i = 0; i < 576; ++i) o[i] = -1;
        for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) {
                const int A = h->conn0[8 * (size_t)e + a], B = h->conn0[8 * (size_t)e + b];
                if (A > B) continue;
                const long long r0 = h->rs[A];
                const int m = h->nup[A];
                const long long rowstart[3] = {r0, r0 + 3 + 3 * m, r0 + 5 + 6LL * m};
                for (int k = 0; k < 3; ++k)
                    for (int l = 0; l < 3; ++l) {
                        long long pos;
                        if (A == B) {
                            if (l < k) continue;
                            pos = rowstart[k] + (l - k);
                        } else {
                            const int r = h->ranks[(size_t)e * 32 + pair_index(std::min(a, b), std::max(a, b))];
                            pos = rowstart[k] + (3 - k) + 3 * r + l;
                        }
                        o[(3 * a + k) * 24 + 3 * b + l] = pos;
                    }
            }
    }
    return 0;
}

namespace ceos {
// Clears the accumulators of one evaluation on stream s.
static int evaluate_prologue(Handle* h, double time, double* dfint, double* dkval, cudaStream_t s) {
    CK(cudaSetDevice(h->device));
    h->time_eval = time;
    CK(cudaMemsetAsync(h->d_status_count, 0, sizeof(int), s));
    CK(cudaMemsetAsync(dfint, 0, sizeof(double) * 3 * (size_t)h->n_nodes, s));
    // FP64 mode accumulates straight into K (zeroed here); the mixed mode writes every K entry
    // from its FP32 node-pair blocks, so K needs no clearing.
    if (dkval && h->precision == CEOS_FP64) CK(cudaMemsetAsync(dkval, 0, sizeof(double) * (size_t)h->nnz, s));
    if (dkval && h->precision == CEOS_MIXED) {
        ++h->epoch;  // the flags of this evaluation's tiles and conversion items
        if (h->ring_dirty) {  // an aborted evaluation may have left partial sums in the blocks
            CK(cudaMemsetAsync(h->d_kblk, 0, (size_t)h->kblk_slots * 12 * sizeof(float), s));
            h->ring_dirty = false;
        }
    }
    return 0;
}

// Elements [e0, e1) = slab `slab` of the host-buffer plan (slab -1: the whole mesh).
static int evaluate_range(Handle* h, double time, const double* dU, double* dfint, double* dkval, cudaStream_t s,
                          int e0, int e1, int slab) {
    const double dt = time - h->time_old;
    const int rc = (h->precision == CEOS_FP64) ? launch_elem<double>(h, dt, dU, dfint, dkval, s, e0, e1, slab)
                                               : launch_elem<float>(h, dt, dU, dfint, dkval, s, e0, e1, slab);
    if (rc && dkval && h->precision == CEOS_MIXED) h->ring_dirty = true;  // blocks may be left unconverted
    return rc;
}

int evaluate_device(Handle* h, double time, const double* dU, double* dfint, double* dkval, cudaStream_t s) {
    int rc = evaluate_prologue(h, time, dfint, dkval, s);
    if (rc) return rc;
    rc = evaluate_range(h, time, dU, dfint, dkval, s, 0, h->n_elem, -1);  // one launch over every slab
    if (rc) return rc;
    h->evaluated = true;
    return 0;
}

// Slab plan of the host-buffer evaluation: n_slabs element ranges; after slab c every node whose
// elements all lie in slabs <= c is final, and the final nodes form the prefix [0, slab_node_end[c])
// of the row order (a running maximum over the nodes of the last slab touching them).  Meshes whose
// numbering follows a sweep (structured or banded) finish a growing prefix after every slab; any
// other numbering simply leaves the copies to the end.
static void plan_slab_bounds(Handle* h) {
    const int kMinElemPerSlab = 16384;
    int ns = std::min(4, h->n_elem / kMinElemPerSlab);
    if (ns < 1) ns = 1;
    // boundaries on whole tiles of kTileE elements: the kernel stages state rows with 16-byte copies
    // from st_old + 32 t, which must stay 16-byte aligned
    h->slab_e.assign(ns + 1, 0);
    for (int c = 1; c < ns; ++c) h->slab_e[c] = (int)((long long)h->n_elem * c / ns / kTileE * kTileE);
    h->slab_e[ns] = h->n_elem;
    std::vector<int> last(h->n_nodes, 0);
    for (int c = 0; c < ns; ++c)
        for (int e = h->slab_e[c]; e < h->slab_e[c + 1]; ++e)
            for (int k = 0; k < 8; ++k) last[h->conn0[(size_t)8 * e + k]] = c;
    h->slab_node_end.assign(ns, 0);
    int run = 0, n = 0;
    for (int c = 0; c < ns; ++c) {
        while (n < h->n_nodes && std::max(run, last[n]) <= c) run = std::max(run, last[n++]);
        h->slab_node_end[c] = n;
    }
    h->slab_node_end[ns - 1] = h->n_nodes;
    h->n_slabs = ns;
}

static int ensure_copy_stream(Handle* h) {
    if (!h->copy_stream && (h->n_slabs > 1 || h->assembly == CEOS_ASSEMBLY_BANDED))
        CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (h->n_slabs > 1 && h->slab_ev.empty()) {
        h->slab_ev.assign(h->n_slabs, nullptr);
        for (auto& ev : h->slab_ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    return 0;
}

// Metadata of conversion items for csr_convert_kernel, two longlong2 per item: {first block, first K
// position}, {first node | nodes << 32, blocks | K values << 32}, checked against the kernel's buffers.
static int upload_conv_meta(Handle* h, const std::vector<ConvItem>& items, void** dst) {
    std::vector<long long> m(4 * std::max<size_t>(items.size(), 1), 0);
    auto bb = [&](int n) { return (long long)n + (h->rs[n] - 6LL * n) / 9; };
    for (size_t j = 0; j < items.size(); ++j) {
        const int n0 = items[j].n0, n1 = items[j].n1, last = n1 - 1;
        const long long nblk = n1 > n0 ? bb(last) + 1 + h->nup[last] - bb(n0) : 0;
        const long long nval = n1 > n0 ? h->rs[last] + 6 + 9LL * h->nup[last] - h->rs[n0] : 0;
        if (n1 - n0 < 1 || n1 - n0 > kBulkNodes || nblk > kBulkBlocks || nval > kBulkStage - 1) {
            h->msg = "conversion item " + std::to_string(j) + " exceeds the conversion buffers";
            return CEOS_E_MESH;
        }
        m[4 * j] = bb(n0);
        m[4 * j + 1] = h->rs[n0];
        m[4 * j + 2] = (long long)n0 | ((long long)(n1 - n0) << 32);
        m[4 * j + 3] = nblk | (nval << 32);
    }
    CK(cudaMalloc(dst, m.size() * sizeof(long long)));
    CK(cudaMemcpy(*dst, m.data(), m.size() * sizeof(long long), cudaMemcpyHostToDevice));
    return 0;
}

// Work queue of the fused element loop + assembly (mixed mode): planned on the host
// (plan_schedule, schedule.cpp), uploaded with the ring of node-pair blocks it sizes.
static int build_schedule(Handle* h) {
    SchedulePlan p;
    // the fused queue, with conversion items sized to the fused kernel's staging
    const int rc = plan_schedule(h->n_nodes, h->n_elem, h->conn0.data(), h->rs.data(), h->nup.data(), h->n_blocks,
                                 h->slab_e, h->slab_node_end, kTileE, h->grid_cap, kStageDoubles, kConvNodes, p);
    if (rc) {
        h->msg = p.err;
        return rc;
    }
    // the two-pass conversion items, sized to the conversion pass's buffers (same cuts at the slab prefixes)
    SchedulePlan p2;
    {
        const int rc2 = plan_schedule(h->n_nodes, h->n_elem, h->conn0.data(), h->rs.data(), h->nup.data(),
                                      h->n_blocks, h->slab_e, h->slab_node_end, kTileE, h->grid_cap, kBulkStage,
                                      kBulkNodes, p2);
        if (rc2) {
            h->msg = p2.err;
            return rc2;
        }
    }
    h->queue = p.queue;
    h->slab_q = p.slab_q;
    h->n_tiles = p.n_tiles;
    h->n_conv = (int)p.conv.size();
    h->ring_blocks = (uint32_t)p.ring_blocks;
    const size_t T = h->n_tiles, J = h->n_conv;
    CK(cudaMalloc(&h->d_queue, h->queue.size() * sizeof(int)));
    CK(cudaMemcpy(h->d_queue, h->queue.data(), h->queue.size() * sizeof(int), cudaMemcpyHostToDevice));
    static_assert(sizeof(ConvItem) == sizeof(int4) && sizeof(TileWait) == sizeof(int2), "item layouts");
    CK(cudaMalloc(&h->d_conv, J * sizeof(int4)));
    CK(cudaMemcpy(h->d_conv, p.conv.data(), J * sizeof(int4), cudaMemcpyHostToDevice));
    h->n_conv2 = (int)p2.conv.size();
    {
        const int mrc = upload_conv_meta(h, p2.conv, &h->d_conv_meta);
        if (mrc) return mrc;
    }
    CK(cudaMalloc(&h->d_tile_wait, T * sizeof(int2)));
    CK(cudaMemcpy(h->d_tile_wait, p.tile_wait.data(), T * sizeof(int2), cudaMemcpyHostToDevice));
    // tile and item flags, then one flag that nothing ever sets (ceos_test_stall_conversion)
    CK(cudaMalloc(&h->d_flags, (T + J + 1) * sizeof(unsigned)));
    CK(cudaMemset(h->d_flags, 0, (T + J + 1) * sizeof(unsigned)));
    h->conv_host = p.conv;
    CK(cudaMalloc(&h->d_ticket, sizeof(unsigned)));
    CK(cudaMalloc(&h->d_sched_err, sizeof(int)));
    CK(cudaMemset(h->d_sched_err, 0, sizeof(int)));
    // two-pass assembly: the items of slab c are those whose last tile lies in slab c (their rows are
    // final after slab c); listed slab by slab, in item order within a slab
    {
        const size_t J2 = h->n_conv2;
        std::vector<int> tile_slab(T, 0);
        for (int c = 0; c < h->n_slabs; ++c)
            for (int t = h->slab_e[c] / kTileE; t < (h->slab_e[c + 1] + kTileE - 1) / kTileE; ++t) tile_slab[t] = c;
        std::vector<int> order;
        order.reserve(J2);
        h->slab_conv.assign(h->n_slabs + 1, 0);
        for (int c = 0; c < h->n_slabs; ++c) {
            h->slab_conv[c] = (int)order.size();
            for (int j = 0; j < (int)J2; ++j)
                if (tile_slab[p2.conv[j].t1] == c) order.push_back(j);
        }
        h->slab_conv[h->n_slabs] = (int)order.size();
        if (order.size() != J2) {
            h->msg = "schedule: conversion items not assigned to slabs";
            return CEOS_E_MESH;
        }
        CK(cudaMalloc(&h->d_conv_order, std::max<size_t>(J2, 1) * sizeof(int)));
        CK(cudaMemcpy(h->d_conv_order, order.data(), J2 * sizeof(int), cudaMemcpyHostToDevice));
    }
    uint32_t pow2 = 1;
    while ((long long)pow2 < h->n_blocks) pow2 <<= 1;
    h->scratch_mask = pow2 - 1;
    // the default two-pass assembly gives every block a slot of its own (ceos_set_assembly resizes)
    h->kblk_slots = h->n_blocks;
    CK(cudaMalloc(&h->d_kblk, (size_t)h->kblk_slots * 12 * sizeof(float)));
    CK(cudaMemset(h->d_kblk, 0, (size_t)h->kblk_slots * 12 * sizeof(float)));
    int per_sm = 1, sms = 148;
    CK(cudaFuncSetAttribute(csr_convert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kBulkSmem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csr_convert_kernel, kThreads, kBulkSmem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    h->conv_grid = sms * std::max(1, per_sm);
    // banded two-pass assembly: bands of two waves of tiles
    {
        BandPlan bp;
        const int band_elems = std::max(1, 2 * h->grid_cap) * kTileE;
        const int brc = plan_bands(h->n_nodes, h->n_elem, h->conn0.data(), h->rs.data(), h->nup.data(), h->n_blocks,
                                   band_elems, kTileE, kBulkStage, kBulkNodes, h->band_depth, bp);
        if (brc) {
            h->msg = bp.err;
            return brc;
        }
        h->n_bands = (int)bp.node_end.size();
        h->band_e = bp.band_e;
        h->band_node_end = bp.node_end;
        h->band_conv = bp.band_conv;
        h->band_ring = (uint32_t)bp.ring_blocks;
        const size_t nbc = bp.conv.size();
        CK(cudaMalloc(&h->d_bconv, std::max<size_t>(nbc, 1) * sizeof(int4)));
        if (nbc) CK(cudaMemcpy(h->d_bconv, bp.conv.data(), nbc * sizeof(int4), cudaMemcpyHostToDevice));
        const int mrc = upload_conv_meta(h, bp.conv, &h->d_bconv_meta);
        if (mrc) return mrc;
    }
    return 0;
}
}  // namespace ceos

extern "C" int ceos_evaluate_device(void* handle, double time, const double* U_device, double* fint_device,
                                    double* kval_device, void* stream) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !U_device || !fint_device) return CEOS_E_ARG;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    return evaluate_device(h, time, U_device, fint_device, kval_device, s);
}

extern "C" int ceos_status(void* handle, int* n_failed) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    if (h->d_sched_err) {  // a bounded wait of the K assembly gave up: K is incomplete
        int err = 0;
        CK(cudaMemcpy(&err, h->d_sched_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) {
            CK(cudaMemset(h->d_sched_err, 0, sizeof(int)));
            h->ring_dirty = true;
            h->msg = "K assembly: a bounded wait exceeded its bound (a dependency wait of the fused assembly, or "
                     "a block copy of the conversion pass)";
            return CEOS_E_CUDA;
        }
    }
    int cnt = 0;
    CK(cudaMemcpy(&cnt, h->d_status_count, sizeof(int), cudaMemcpyDeviceToHost));
    if (n_failed) *n_failed = cnt;
    if (!cnt) return 0;
    std::vector<uint8_t> st(h->n_elem);
    CK(cudaMemcpy(st.data(), h->d_elem_status, h->n_elem, cudaMemcpyDeviceToHost));
    int worst = 0;
    for (uint8_t v : st) worst |= v;
    if (worst & 1) return 1;
    if (worst & 2) return 2;
    return 3;
}

extern "C" int ceos_evaluate(void* handle, double time, const double* U, double* fint, double* kval, int* n_failed) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !U || !fint) return CEOS_E_ARG;
    CK(cudaSetDevice(h->device));
    cudaStream_t s = h->stream;
    const size_t nd = 3 * (size_t)h->n_nodes;
    {
        const int rc = ensure_copy_stream(h);
        if (rc) return rc;
    }
    CK(cudaMemcpyAsync(h->d_U, U, nd * sizeof(double), cudaMemcpyHostToDevice, s));
    double* dk = kval ? h->d_kval : nullptr;
    int rc = evaluate_prologue(h, time, h->d_fint, dk, s);
    if (rc) return rc;
    if (kval && h->precision == CEOS_MIXED && h->assembly == CEOS_ASSEMBLY_BANDED) {
        // the bands copy their finished rows to the host on copy_stream as they go
        h->copy_f = fint;
        h->copy_k = kval;
        rc = evaluate_range(h, time, h->d_U, h->d_fint, dk, s, 0, h->n_elem, -1);
        h->copy_f = h->copy_k = nullptr;
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->copy_stream));
    } else if (h->n_slabs == 1) {
        rc = evaluate_range(h, time, h->d_U, h->d_fint, dk, s, 0, h->n_elem, -1);
        if (rc) return rc;
        CK(cudaMemcpyAsync(fint, h->d_fint, nd * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (kval) CK(cudaMemcpyAsync(kval, h->d_kval, (size_t)h->nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
    } else {
        // slab c computes on s; the rows it finished travel to the host on copy_stream meanwhile
        int n_done = 0;
        for (int c = 0; c < h->n_slabs; ++c) {
            const int n_end = h->slab_node_end[c];
            rc = evaluate_range(h, time, h->d_U, h->d_fint, dk, s, h->slab_e[c], h->slab_e[c + 1], c);
            if (rc) return rc;
            if (n_end > n_done) {
                CK(cudaEventRecord(h->slab_ev[c], s));
                CK(cudaStreamWaitEvent(h->copy_stream, h->slab_ev[c], 0));
                CK(cudaMemcpyAsync(fint + 3 * (size_t)n_done, h->d_fint + 3 * (size_t)n_done,
                                   3 * (size_t)(n_end - n_done) * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->copy_stream));
                if (kval) {
                    const long long k0 = h->rs[n_done], k1 = n_end < h->n_nodes ? h->rs[n_end] : h->nnz;
                    CK(cudaMemcpyAsync(kval + k0, h->d_kval + k0, (size_t)(k1 - k0) * sizeof(double),
                                       cudaMemcpyDeviceToHost, h->copy_stream));
                }
            }
            n_done = n_end;
        }
        CK(cudaStreamSynchronize(h->copy_stream));
    }
    h->evaluated = true;
    CK(cudaStreamSynchronize(s));
    return ceos_status(handle, n_failed);
}

extern "C" int ceos_commit_state(void* handle) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    // The state written by the last evaluation becomes the committed one (the reference copies
    // new into old; swapping the buffers is the same as long as an evaluation happened since the
    // last commit, which the flag guarantees).
    if (h->evaluated) {
        h->cur_old = 1 - h->cur_old;
        h->evaluated = false;
        CK(cudaSetDevice(h->device));
        if (h->nstate)
            CK(cudaMemcpyAsync(h->d_state[1 - h->cur_old], h->d_state[h->cur_old], h->state_bytes(),
                               cudaMemcpyDeviceToDevice, h->stream));
    }
    h->time_old = h->time_eval;
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

extern "C" int ceos_set_committed_time(void* handle, double t) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    h->time_old = t;
    h->time_eval = t;
    return 0;
}

extern "C" int ceos_last_error(void* handle, int* elem_ids, int max_ids, char* msg, int msg_len) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    std::vector<uint8_t> st(h->n_elem);
    CK(cudaMemcpy(st.data(), h->d_elem_status, h->n_elem, cudaMemcpyDeviceToHost));
    int n = 0, worst = 0;
    for (int e = 0; e < h->n_elem; ++e)
        if (st[e]) {
            if (elem_ids && n < max_ids) elem_ids[n] = e + 1;
            ++n;
            worst |= st[e];
        }
    if (msg && msg_len > 0) {
        std::string m;
        if (!n) m = h->msg.empty() ? "no error" : h->msg;
        else if (worst & 1) m = "Determinant of the Jacobian Matrix <= 0.0d0 in " + std::to_string(n) + " element(s)";
        else if (worst & 2) m = "Max Iteration in Local Newton-Raphson in " + std::to_string(n) + " element(s)";
        else m = "Non-finite stress in " + std::to_string(n) + " element(s)";
        std::strncpy(msg, m.c_str(), msg_len - 1);
        msg[msg_len - 1] = 0;
    }
    return n;
}

// Deformation gradient at every Gauss point from device displacements: F [9][8 n_elem] (row-major
// components, point q = gp * n_elem + e), F = I + dU/dX with the Hexa8 shape functions.
__global__ void gp_deformation_kernel(int n_elem, const double* X, const double* U, const int* conn0, double* F) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= 8LL * n_elem) return;
    const int gp = (int)(q / n_elem), e = (int)(q - (long long)gp * n_elem);
    double JX[3][3] = {}, Xn[8][3], Un[8][3];
    for (int n = 0; n < 8; ++n) {
        const int a = conn0[(size_t)8 * e + n];
        for (int d = 0; d < 3; ++d) { Xn[n][d] = X[3 * (size_t)a + d]; Un[n][d] = U[3 * (size_t)a + d]; }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) JX[i][j] += c_dN[gp][n][i] * Xn[n][j];
    }
    const double det = det3(JX);
    double Ji[3][3];
    inv3(JX, det, Ji);
    double Fm[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int n = 0; n < 8; ++n) {
        double gX[3];
        for (int j = 0; j < 3; ++j) gX[j] = Ji[j][0] * c_dN[gp][n][0] + Ji[j][1] * c_dN[gp][n][1] + Ji[j][2] * c_dN[gp][n][2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Fm[i][j] += Un[n][i] * gX[j];
    }
    const long long ld = 8LL * n_elem;
    for (int k = 0; k < 9; ++k) F[k * ld + q] = Fm[k / 3][k % 3];
}

extern "C" int ceos_gp_deformation_device(void* handle, const double* dU, double* dF, void* stream) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !dU || !dF) return CEOS_E_ARG;
    CK(cudaSetDevice(h->device));
    const long long n = 8LL * h->n_elem;
    gp_deformation_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        h->n_elem, h->d_X, dU, h->d_conn, dF);
    CK(cudaGetLastError());
    return 0;
}

// Replace the per-element parameters of a handle created with per_element materials:
// params [n_elem][n_params] (element-major, as at creation).
extern "C" int ceos_update_params(void* handle, const double* params) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !params || h->param_mode != 1) return CEOS_E_ARG;
    CK(cudaSetDevice(h->device));
    const size_t E = h->n_elem, np = h->n_params;
    std::vector<double> P(np * E);
    for (size_t e = 0; e < E; ++e)
        for (size_t k = 0; k < np; ++k) P[k * E + e] = params[e * np + k];
    h->host_params = P;
    CK(cudaStreamSynchronize(h->stream));
    if (h->precision == CEOS_FP64) {
        CK(cudaMemcpy(h->d_params, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(P.begin(), P.end());
        CK(cudaMemcpy(h->d_params, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return 0;
}

// Device pointer of the committed Gauss-point state ([nvars][8][ld], FP64 or FP32 by precision
// mode), e.g. for an external material to write the stress and tangent the loop reads.
extern "C" int ceos_state_device(void* handle, void** ptr, long long* ld, int* is_f32) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !ptr) return CEOS_E_ARG;
    *ptr = h->d_state[h->cur_old];
    if (ld) *ld = h->ld;
    if (is_f32) *is_f32 = h->precision == CEOS_MIXED ? 1 : 0;
    return 0;
}

extern "C" int ceos_state_size(void* handle, int* nvars) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !nvars) return CEOS_E_ARG;
    *nvars = h->nstate;
    return 0;
}

extern "C" int ceos_get_state(void* handle, int which, double* out) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !out) return CEOS_E_ARG;
    if (!h->nstate) return 0;
    const int buf = which ? 1 - h->cur_old : h->cur_old;
    const size_t n = (size_t)h->nstate * 8 * h->ld;
    std::vector<double> tmp(n);
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (h->precision == CEOS_FP64) {
        CK(cudaMemcpy(tmp.data(), h->d_state[buf], n * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> f(n);
        CK(cudaMemcpy(f.data(), h->d_state[buf], n * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) tmp[i] = f[i];
    }
    // device [v][gp][e] (leading dimension ld) -> host [e][gp][v]
    const int E = h->n_elem, V = h->nstate;
    const size_t LD = h->ld;
    for (int v = 0; v < V; ++v)
        for (int g = 0; g < 8; ++g)
            for (int e = 0; e < E; ++e) out[((size_t)e * 8 + g) * V + v] = tmp[((size_t)v * 8 + g) * LD + e];
    return 0;
}

extern "C" int ceos_set_state(void* handle, int which, const double* in) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !in) return CEOS_E_ARG;
    if (!h->nstate) return 0;
    const int buf = which ? 1 - h->cur_old : h->cur_old;
    const int E = h->n_elem, V = h->nstate;
    const size_t LD = h->ld;
    const size_t n = (size_t)V * 8 * LD;
    std::vector<double> tmp(n, 0.0);
    for (int v = 0; v < V; ++v)
        for (int g = 0; g < 8; ++g)
            for (int e = 0; e < E; ++e) tmp[((size_t)v * 8 + g) * LD + e] = in[((size_t)e * 8 + g) * V + v];
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (h->precision == CEOS_FP64) {
        CK(cudaMemcpy(h->d_state[buf], tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(tmp.begin(), tmp.end());
        CK(cudaMemcpy(h->d_state[buf], f.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    }
    return 0;
}

extern "C" int ceos_set_options(void* handle, int options) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    h->options = options;
    if ((options & CEOS_OPT_TIME_KERNELS) && !h->ev_k0) {
        CK(cudaSetDevice(h->device));
        CK(cudaEventCreate(&h->ev_k0));
        CK(cudaEventCreate(&h->ev_k1));
        CK(cudaEventCreate(&h->ev_k2));
    }
    if ((options & CEOS_OPT_STORE_STRESS) && !h->d_gp_stress) {
        CK(cudaSetDevice(h->device));
        CK(cudaMalloc(&h->d_gp_stress, (size_t)6 * 8 * h->n_elem * h->elem_bytes()));
    }
    return 0;
}

extern "C" int ceos_test_stall_conversion(void* handle, int item, int on) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || h->precision != CEOS_MIXED || item < 0 || item >= h->n_conv) return CEOS_E_ARG;
    ConvItem c = h->conv_host[item];
    if (on) c.t0 = c.t1 = h->n_tiles + h->n_conv;  // the tile-flag index of the sentinel flag
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(static_cast<int4*>(h->d_conv) + item, &c, sizeof(int4), cudaMemcpyHostToDevice));
    return 0;
}

extern "C" int ceos_launch_count(void* handle, int tangent, int* n_launches) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !n_launches) return CEOS_E_ARG;
    int n = 1;  // the element loop
    if (tangent && h->precision == CEOS_MIXED) {
        if (h->assembly == CEOS_ASSEMBLY_TWO_PASS) {
            n = 1 + (h->n_conv2 > 0 ? 1 : 0);
        } else if (h->assembly == CEOS_ASSEMBLY_BANDED) {
            n = h->n_bands;
            for (int c = 0; c < h->n_bands; ++c) n += h->band_conv[c + 1] > h->band_conv[c] ? 1 : 0;
        }
    }
    *n_launches = n;
    return 0;
}

extern "C" int ceos_set_assembly(void* handle, int mode) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || (mode != CEOS_ASSEMBLY_TWO_PASS && mode != CEOS_ASSEMBLY_FUSED && mode != CEOS_ASSEMBLY_BANDED))
        return CEOS_E_ARG;
    if (h->precision == CEOS_MIXED && h->d_kblk) {
        // slots the mode uses: every block, or a power-of-two ring (a ring of at least n_blocks slots
        // indexes blocks directly, so n_blocks of them suffice)
        const long long ring = mode == CEOS_ASSEMBLY_FUSED ? (long long)h->ring_blocks : (long long)h->band_ring;
        const long long need = mode == CEOS_ASSEMBLY_TWO_PASS ? h->n_blocks : std::min(ring, h->n_blocks);
        if (need != h->kblk_slots) {  // the new slots exist before the old ones go: a failure changes nothing
            CK(cudaSetDevice(h->device));
            CK(cudaStreamSynchronize(h->stream));
            float* fresh = nullptr;
            CK(cudaMalloc(&fresh, (size_t)need * 12 * sizeof(float)));
            if (cudaMemset(fresh, 0, (size_t)need * 12 * sizeof(float)) != cudaSuccess) {
                cudaFree(fresh);
                h->msg = "ceos_set_assembly: clearing the block slots failed";
                return CEOS_E_CUDA;
            }
            cudaFree(h->d_kblk);
            h->d_kblk = fresh;
            h->kblk_slots = need;
            h->ring_dirty = false;
        }
    }
    h->assembly = mode;  // every mode leaves the slots it uses at zero after an evaluation
    return 0;
}

extern "C" int ceos_kernel_time(void* handle, float* ms) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !ms || !h->ev_k0) return CEOS_E_ARG;
    CK(cudaEventSynchronize(h->ev_k2));
    CK(cudaEventElapsedTime(&ms[0], h->ev_k0, h->ev_k1));
    CK(cudaEventElapsedTime(&ms[1], h->ev_k1, h->ev_k2));
    return 0;
}

extern "C" int ceos_gp_stress(void* handle, double* out) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !out || !h->d_gp_stress) return CEOS_E_ARG;
    const int E = h->n_elem;
    const size_t n = (size_t)6 * 8 * E;
    std::vector<double> tmp(n);
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (h->precision == CEOS_FP64) {
        CK(cudaMemcpy(tmp.data(), h->d_gp_stress, n * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> f(n);
        CK(cudaMemcpy(f.data(), h->d_gp_stress, n * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) tmp[i] = f[i];
    }
    for (int k = 0; k < 6; ++k)
        for (int g = 0; g < 8; ++g)
            for (int e = 0; e < E; ++e) out[((size_t)e * 8 + g) * 6 + k] = tmp[((size_t)k * 8 + g) * E + e];
    return 0;
}

extern "C" void ceos_destroy(void* handle) {
    Handle* h = static_cast<Handle*>(handle);
    delete h;
}

// ---------------------------------------------------------------------------------------
// Device allocation (Handle::allocate_device)
// ---------------------------------------------------------------------------------------
namespace ceos {

int Handle::allocate_device(const ceos_mesh* mesh, const ceos_material* mats, int n_mat) {
    Handle* h = this;
    const size_t N = n_nodes, E = n_elem;
    ld = (n_elem + 31) / 32 * 32;
    conn0.resize(8 * E);
    for (size_t i = 0; i < 8 * E; ++i) conn0[i] = mesh->conn[i] - 1;
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&d_X, 3 * N * sizeof(double)));
    CK(cudaMemcpy(d_X, mesh->X, 3 * N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&d_U, 3 * N * sizeof(double)));
    CK(cudaMemset(d_U, 0, 3 * N * sizeof(double)));
    CK(cudaMalloc(&d_fint, 3 * N * sizeof(double)));
    CK(cudaMalloc(&d_kval, (size_t)nnz * sizeof(double)));
    CK(cudaMalloc(&d_conn, 8 * E * sizeof(int)));
    CK(cudaMemcpy(d_conn, conn0.data(), 8 * E * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&d_rs, N * sizeof(long long)));
    CK(cudaMemcpy(d_rs, rs.data(), N * sizeof(long long), cudaMemcpyHostToDevice));
    if (precision == CEOS_MIXED) {  // first node-pair block of each node: n + (rs[n] - 6n) / 9
        std::vector<long long> blk0(N);
        for (size_t n = 0; n < N; ++n) blk0[n] = (long long)n + (rs[n] - 6LL * (long long)n) / 9;
        CK(cudaMalloc(&d_blk0, N * sizeof(long long)));
        CK(cudaMemcpy(d_blk0, blk0.data(), N * sizeof(long long), cudaMemcpyHostToDevice));
    }
    if (precision == CEOS_MIXED) {
        // reference geometry of every Gauss point for the FP32 element arithmetic: J_X^-1 and det J_X
        // in FP64 (J_X = sum_n dN_n/dxi (x) X_n, ModElement.f90:1210-1300), rounded once to FP32
        double tab[8][8][3];
        hexa8_dN_table(tab);
        std::vector<float> G((size_t)10 * 8 * ld, 0.f);
        for (size_t e = 0; e < E; ++e) {
            const int* cn = conn0.data() + 8 * e;
            for (int gp = 0; gp < 8; ++gp) {
                double J[3][3] = {};
                for (int n = 0; n < 8; ++n)
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) J[i][j] += tab[gp][n][i] * mesh->X[3 * (size_t)cn[n] + j];
                const double d = det3(J);
                double Ji[3][3] = {};
                if (std::fabs(d) > 1e-300) inv3(J, d, Ji);
                for (int k = 0; k < 9; ++k) G[((size_t)k * 8 + gp) * ld + e] = (float)Ji[k / 3][k % 3];
                G[((size_t)9 * 8 + gp) * ld + e] = (float)d;
            }
        }
        CK(cudaMalloc(&d_jxi, G.size() * sizeof(float)));
        CK(cudaMemcpy(d_jxi, G.data(), G.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&d_nup, N * sizeof(int)));
    CK(cudaMemcpy(d_nup, nup.data(), N * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&d_ranks, E * 32));
    CK(cudaMemcpy(d_ranks, ranks.data(), E * 32, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&d_elem_status, E));
    CK(cudaMemset(d_elem_status, 0, E));
    CK(cudaMalloc(&d_status_count, sizeof(int)));
    CK(cudaMemset(d_status_count, 0, sizeof(int)));
    // parameters
    const size_t eb = elem_bytes();
    std::vector<double> P;
    bool any_per_element = false;
    for (int k = 0; k < n_mat; ++k) any_per_element |= mats[k].per_element != 0;
    if (any_per_element) {
        param_mode = 1;
        P.assign((size_t)n_params * E, 0.0);
        for (size_t e = 0; e < E; ++e) {
            const int mid = mesh->mat_id ? mesh->mat_id[e] : 0;
            if (mid < 0 || mid >= n_mat) { msg = "bad mat_id"; return CEOS_E_MESH; }
            const ceos_material& m = mats[mid];
            const double* src = m.per_element ? m.params + e * (size_t)m.n_params : m.params;
            for (int k = 0; k < n_params; ++k) P[(size_t)k * E + e] = src[k];
        }
    } else if (n_mat == 1) {
        param_mode = 0;
        P.assign(mats[0].params, mats[0].params + n_params);
    } else {
        param_mode = 2;
        P.resize((size_t)n_mat * n_params);
        for (int m = 0; m < n_mat; ++m)
            for (int k = 0; k < n_params; ++k) P[(size_t)m * n_params + k] = mats[m].params[k];
        std::vector<int> mid(E);
        for (size_t e = 0; e < E; ++e) {
            mid[e] = mesh->mat_id ? mesh->mat_id[e] : 0;
            if (mid[e] < 0 || mid[e] >= n_mat) { msg = "bad mat_id"; return CEOS_E_MESH; }
        }
        CK(cudaMalloc(&d_mat_id, E * sizeof(int)));
        CK(cudaMemcpy(d_mat_id, mid.data(), E * sizeof(int), cudaMemcpyHostToDevice));
    }
    host_params = P;
    // node-pair blocks of the FP32 assembly: one diagonal block per node, one per upper neighbour
    // (the ring that holds them is sized with the schedule, build_schedule)
    n_blocks = (long long)N + (nnz - 6LL * (long long)N) / 9;
    // state variables actually used (the Prony model reads/writes only nb of its 4 branch slots)
    ns_used = nstate;
    if (model == M_VISCO_PRONY && param_mode == 0) ns_used = 6 + 6 * std::max(0, std::min(4, (int)P[2]));
    CK(cudaMalloc(&d_params, P.size() * eb));
    if (precision == CEOS_FP64) {
        CK(cudaMemcpy(d_params, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(P.begin(), P.end());
        CK(cudaMemcpy(d_params, f.data(), P.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    // state: virgin state in both buffers, device layout [v][gp][e]
    if (nstate) {
        std::vector<double> init(nstate);
        model_init_state(model, init.data());
        std::vector<double> S((size_t)nstate * 8 * ld);
        for (int v = 0; v < nstate; ++v)
            std::fill(S.begin() + (size_t)v * 8 * ld, S.begin() + (size_t)(v + 1) * 8 * ld, init[v]);
        for (int b = 0; b < 2; ++b) {
            CK(cudaMalloc(&d_state[b], state_bytes()));
            if (precision == CEOS_FP64) {
                CK(cudaMemcpy(d_state[b], S.data(), state_bytes(), cudaMemcpyHostToDevice));
            } else {
                std::vector<float> f(S.begin(), S.end());
                CK(cudaMemcpy(d_state[b], f.data(), state_bytes(), cudaMemcpyHostToDevice));
            }
        }
    }
    return 0;
}

Handle::~Handle() {
    if (stream) cudaStreamSynchronize(stream);
    void* ptrs[] = {d_X, d_jxi, d_U, d_fint, d_kval, d_conn, d_rs, d_blk0, d_nup, d_ranks, d_elem_status, d_status_count,
                    d_params, d_mat_id, d_state[0], d_state[1], d_gp_stress, d_kblk, d_queue, d_conv,
                    d_tile_wait, d_flags, d_ticket, d_sched_err, d_conv_order, d_bconv, d_conv_meta, d_bconv_meta};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (ev_k0) cudaEventDestroy(ev_k0);
    if (ev_k1) cudaEventDestroy(ev_k1);
    if (ev_k2) cudaEventDestroy(ev_k2);
    for (cudaEvent_t ev : slab_ev)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : ev_band)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : ev_bconv)
        if (ev) cudaEventDestroy(ev);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (band_stream) cudaStreamDestroy(band_stream);
    if (conv_stream) cudaStreamDestroy(conv_stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (stream) cudaStreamDestroy(stream);
}

}  // namespace ceos
