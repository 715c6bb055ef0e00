// ceos_handle.h -- the state behind one ceos_gpu.h handle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ceos_gpu.h"
#include "schedule.h"

namespace ceos {

struct Handle {
    // mesh and pattern (host copies)
    int n_nodes = 0, n_elem = 0, precision = 0, device = 0, model = 0, n_params = 0, nstate = 0;
    int ld = 0;       // leading dimension of state arrays: n_elem rounded up to 32
    int ns_used = 0;  // state variables the kernel reads and writes
    long long nnz = 0;
    std::vector<int> conn0;               // [8*n_elem] 0-based
    std::vector<long long> up_ptr;        // upper-neighbour lists (CSR over nodes)
    std::vector<int> up_list;
    std::vector<long long> rs;            // CSR position of row 3n
    std::vector<int> nup;                 // number of upper neighbours of node n
    std::vector<uint8_t> ranks;           // [n_elem*32] slot ranks per local pair
    std::vector<double> host_params;
    int param_mode = 0;
    // device buffers
    cudaStream_t stream = nullptr;
    double *d_X = nullptr, *d_U = nullptr, *d_fint = nullptr, *d_kval = nullptr;
    int* d_conn = nullptr;
    long long* d_rs = nullptr;
    long long* d_blk0 = nullptr;          // mixed mode: first node-pair block of each node
    int* d_nup = nullptr;
    uint32_t* d_ranks = nullptr;
    uint8_t* d_elem_status = nullptr;
    int* d_status_count = nullptr;
    void* d_params = nullptr;
    int* d_mat_id = nullptr;
    void* d_state[2] = {nullptr, nullptr};
    void* d_gp_stress = nullptr;
    float* d_jxi = nullptr;               // mixed mode: [10][8][ld] J_X^-1 and det J_X per Gauss point (FP32 of FP64)
    float* d_kblk = nullptr;              // mixed mode: FP32 node-pair block slots, kblk_slots of them: every
                                          // block (two-pass) or the ring of the fused / banded assembly
    long long kblk_slots = 0;
    long long n_blocks = 0;
    int assembly = CEOS_ASSEMBLY_TWO_PASS;  // mixed mode with a tangent: two-pass or fused assembly
    uint32_t scratch_mask = 0;            // two-pass: power of two minus one, >= every block index
    std::vector<int> slab_conv;           // [n_slabs + 1] two-pass: conversion items of slab c are
                                          // d_conv_order[slab_conv[c] .. slab_conv[c + 1])
    int* d_conv_order = nullptr;
    int conv_grid = 148;                  // CTAs of a conversion launch
    // banded two-pass assembly: element bands on two alternating streams, each band's conversion on
    // a third; the blocks live in a ring of band_ring slots (see plan_bands, schedule.h)
    int n_bands = 0;
    std::vector<int> band_e, band_node_end, band_conv;
    void* d_bconv = nullptr;              // int4 [band_conv[n_bands]] conversion items of the bands
    void* d_bconv_meta = nullptr;         // longlong2 [2 band_conv[n_bands]] their conversion-pass metadata
    uint32_t band_ring = 0;
    int band_depth = 3;                   // element band c starts after the conversion of band c - depth
    cudaStream_t band_stream = nullptr;   // odd element bands (even ones run on the caller's stream)
    cudaStream_t conv_stream = nullptr;   // conversions, highest priority
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_band, ev_bconv;
    double* copy_f = nullptr;             // host-buffer call with the banded assembly: f_int and K rows
    double* copy_k = nullptr;             // go to these host arrays band by band on copy_stream
    // fused assembly schedule (mixed mode with a tangent): a queue of element tiles and CSR
    // conversion items, split at the element slabs of the host-buffer evaluation
    std::vector<int> queue;               // >= 0 tile, < 0 conversion item -(j+1)
    std::vector<ConvItem> conv_host;      // the planned conversion items (host copy)
    std::vector<int> slab_q;              // [n_slabs + 1] queue position where slab c starts
    int n_tiles = 0, n_conv = 0;
    uint32_t ring_blocks = 0;             // power of two; block b lives in slot b & (ring_blocks - 1)
    int* d_queue = nullptr;
    void* d_conv = nullptr;               // int4 [n_conv] {first node, end node, first tile, last tile}
    int n_conv2 = 0;                      // two-pass conversion items (planned to the conversion pass's bounds)
    void* d_conv_meta = nullptr;          // longlong2 [2 n_conv2] their metadata for the conversion pass
    void* d_tile_wait = nullptr;          // int2 [n_tiles] conversion items that last used the tile's slots
    unsigned* d_flags = nullptr;          // [n_tiles] tile done, [n_conv] conversion done (epoch values)
    unsigned* d_ticket = nullptr;         // work counter of the running launch
    int* d_sched_err = nullptr;           // a bounded wait gave up
    unsigned epoch = 0;
    bool ring_dirty = false;              // an aborted evaluation may have left non-zero slots
    int cur_old = 0;                      // index of the committed state buffer
    bool evaluated = false;
    double time_old = 0.0, time_eval = 0.0;
    int options = 0;
    cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr, ev_k2 = nullptr;
    // host-buffer evaluation in element slabs: after slab c the node rows [0, slab_node_end[c]) are final
    // and go to the host on copy_stream while the next slabs compute
    int n_slabs = 0;                      // 0: plan not built yet
    std::vector<int> slab_e;              // [n_slabs + 1] element boundaries
    std::vector<int> slab_node_end;       // [n_slabs] final node-row prefix after each slab
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> slab_ev;
    int grid_cap = 148, blocks_per_sm = 1;
    std::string msg;
    // host analysis driver: per-substep result callback and the starting U of a restart
    ceos_step_callback step_cb = nullptr;
    void* step_user = nullptr;
    std::vector<double> U_start;          // empty: start from U = 0
    bool device_newton = false;           // ceos_analysis keeps K on the device and solves by PCG
    double lin_tol = 1e-12;
    int lin_max_iter = 20000;

    size_t elem_bytes() const { return precision == CEOS_FP64 ? sizeof(double) : sizeof(float); }
    size_t state_bytes() const { return (size_t)nstate * 8 * ld * elem_bytes(); }
    int allocate_device(const ceos_mesh* mesh, const ceos_material* mats, int n_mat);
    ~Handle();
};

int evaluate_device(Handle* h, double time, const double* dU, double* dfint, double* dkval, cudaStream_t s);

}  // namespace ceos
