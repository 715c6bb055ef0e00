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
//             node pairs it owns, then scatters them into f_int and K.
// Warp-uniform roles (gp or b is the warp index) keep control flow convergent; the shared
// layouts put the element index innermost so every shared access is conflict-free.
//
// Kernels using these phases:
//   element_loop_kernel<T, MODEL, SCATTER>: static tile schedule.  SCATTER_CSR64: K by FP64
//     atomics straight into the CSR values (CEOS_FP64), or no K (an evaluation without tangent).
//     SCATTER_RING (CEOS_MIXED with a tangent, two-pass assembly): K by 16-byte FP32 vector
//     reductions into node-pair blocks (3 rows x 4 floats per node pair) in a scratch array that
//     holds every block; csr_convert_kernel then turns finished blocks into the FP64 CSR rows.
//   element_assemble_kernel<MODEL>: CEOS_MIXED with a tangent, fused assembly.  K accumulates in FP32 node-pair
//     blocks (3 rows x 4 floats per node pair) by 16-byte vector reductions, and the same launch
//     turns finished blocks into the FP64 CSR rows.  The blocks live in a ring of 2^k blocks
//     (block b in slot b & mask) sized to stay in L2, so the FP32 accumulation never travels to
//     HBM: HBM sees the inputs once and the FP64 K once.  The CTAs take work from a queue built on
//     the host: element tiles, and conversion items (a run of node rows) placed after the last
//     tile that touches those rows.  A conversion item waits until those tiles have reduced;
//     a tile waits until the items that last used its ring slots have written their rows and
//     zeroed the slots.  Every wait is for work earlier in the queue (the host checks this), so
//     the earliest unfinished item can always proceed; each wait is also bounded and reports a
//     scheduling error instead of hanging.
#pragma once
#include "ceos_common.cuh"
#include "materials.cuh"
#include "visco_var.cuh"

namespace ceos {

constexpr int kTileE = 32;
constexpr int kThreads = 256;
constexpr int kEndItem = -0x7fffffff - 1;   // queue sentinel: no more work
constexpr unsigned long long kWaitNs = 200ull * 1000 * 1000;  // bound of every flag wait: 200 ms

// dN/dxi of the 8 nodes at the 8 Gauss points (ModElementHexa8.f90:211-268, points :278-329).
// (defined once: this header is included by a single translation unit)
__constant__ double c_dN[8][8][3];
__constant__ float c_dNf[8][8][3];  // the same table rounded to FP32 for the mixed-precision path

template <typename T>
CEOS_D T dN_at(int gp, int n, int i) {
    if constexpr (sizeof(T) == 4) return c_dNf[gp][n][i];
    else return c_dN[gp][n][i];
}

template <typename T>
struct ElemArgs {
    int n_elem;
    int e_begin, e_end;     // element range of this launch (static schedule)
    const double* X;        // [3*n_nodes] reference coordinates (CoordX)
    const float* jxi;       // FP32 mode: [10][8][ld] J_X^-1 (row-major, 9) and det J_X of every Gauss point
    const double* U;        // [3*n_nodes] displacements, DOF 3n+d
    const int* conn;        // [n_elem*8] 0-based node ids
    const long long* rs;    // [n_nodes] CSR position of the first entry of row 3n (0-based); blocked
                            // assembly: the first node-pair block of node n instead
    const int* nup;         // [n_nodes] number of neighbour nodes with a larger id
    const uint32_t* ranks;  // [n_elem*8] 28 uint8 slot ranks per element (32 bytes)
    double* fint;           // [3*n_nodes]
    double* kval;           // [nnz] or nullptr (no tangent)
    const T* st_old;        // [nstate][8][ld]
    T* st_new;
    int ld;                 // leading dimension of the state arrays (n_elem rounded up to 32)
    int ns_used;            // state variables the model reads and writes
    int n_pe;               // per-element parameters staged per tile (n_params when param_mode 1, else 0)
    const T* params;        // see param_mode
    int param_mode;         // 0 uniform (pu[]); 1 per element params[k*n_elem+e]; 2 per material
    int n_params;
    const int* mat_id;      // per material: params[mat_id[e]*n_params+k]
    T pu[12];               // uniform parameters (kernel-argument space: broadcast reads)
    T ebr[4];               // Prony relaxation factors exp(-dt/(2 tau_a)) when parameters are uniform
    double dt;
    uint8_t* elem_status;   // [n_elem]
    int* status_count;      // failed elements
    T* gp_stress;           // [6][8][n_elem] or nullptr
    // ---- mixed-precision K assembly (two-pass element pass and conversion; fused kernel) ----
    float* kblk;            // FP32 node-pair blocks, 12 floats each (3 rows of 4; a diagonal block packs its upper
                            // 6 entries into the first 6 floats), zero between evaluations
    uint32_t ring_mask;     // block b lives in slot b & ring_mask (two-pass: every block its own slot)
    const long long* csr_rs;   // [n_nodes] CSR position of row 3n (0-based)
    const int* queue;       // work items: >= 0 element tile, < 0 conversion item -(j+1)
    int q_begin, q_end;     // this launch's part of the queue
    unsigned* ticket;       // work counter, zero at launch
    unsigned* tile_done;    // [n_tiles] = epoch once the tile's reductions are complete
    unsigned* conv_done;    // [n_conv] = epoch once the item's rows are written and slots zeroed
    unsigned epoch;
    const int4* conv;       // [n_conv] {first node, end node, first tile, last tile} of an item
    const longlong2* conv_meta;  // [2 n_conv] conversion pass: {first block, first K position},
                                 // {first node | nodes << 32, blocks | K values << 32} of an item
    const int2* tile_wait;  // [n_tiles] items [x, y) that last used the ring slots of the tile
    int* sched_err;         // set when a wait exceeds its bound
};

// Dynamic shared-memory layout of one CTA.  Arrays indexed [..][e] with the element index
// innermost, so that 32 lanes (32 consecutive elements) access consecutive words or 16-byte
// vectors: every access is bank-conflict free.  Node data and state of the NEXT tile are
// prefetched with cp.async while the current tile computes (software pipeline).
template <typename T>
struct SmemLayout {
    size_t g, ds, st, x, u, rs, nup, node, ranks, status, kd, pe, total;
    CEOS_HD SmemLayout(int ns, int npe) {
        size_t o = 0;
        auto take = [&](size_t bytes) { size_t r = o; o += (bytes + 15) & ~size_t(15); return r; };
        g = take(sizeof(T) * 8 * 8 * kTileE * 4);        // [gp][node][e][4]: grad N (current)
        ds = take(sizeof(T) * 8 * 7 * kTileE * 4);       // [gp][quad][e][4]: w detJ (D upper 21, sigma 6)
        st = take(sizeof(T) * (size_t)(ns > 0 ? ns : 1) * 8 * kTileE);  // [v][gp][e]: committed state
        x = take(sizeof(double) * 8 * kTileE * 3);     // [node][e][3] staged X (FP64)
        u = take(sizeof(double) * 8 * kTileE * 3);     // [node][e][3] staged U (FP64)
        rs = take(sizeof(long long) * 2 * 8 * kTileE);  // double-buffered [buf][node][e]
        nup = take(sizeof(int) * 2 * 8 * kTileE);
        node = take(sizeof(int) * 2 * 8 * kTileE);
        ranks = take(sizeof(uint32_t) * 2 * kTileE * 8); // [buf][e][8]
        status = take(sizeof(int) * kTileE);
        kd = take(sizeof(double) * kTileE);              // [e] Mean Dilatation: d2psi/dJbar2 / V0
        pe = take(sizeof(T) * (size_t)(npe > 0 ? npe : 1) * kTileE);  // [k][e] per-element parameters
        total = o;
    }
};
// The fused kernel's conversion of a run of CSR rows stages its FP64 values in the g and ds regions
// (unused between tiles), followed by a table of its nodes (first block, first K value, upper
// neighbours), so an item it converts holds at most kConvNodes nodes and kStageDoubles K values.  The
// items are planned to the tighter bounds of the conversion pass (kBulkNodes, kBulkStage), which
// both kernels then hold.
constexpr int kConvNodes = 256;
constexpr int kStageRegion = (int)(sizeof(float) * 8 * 8 * kTileE * 4 + sizeof(float) * 8 * 7 * kTileE * 4);
constexpr int kStageDoubles = (kStageRegion - 3 * kConvNodes * (int)sizeof(int)) / 8 - 2;
static_assert((kStageDoubles + 2) * 8 + 3 * kConvNodes * (int)sizeof(int) <= kStageRegion, "conversion staging");

template <typename T>
struct SmemPtrs {
    T *g, *ds, *st, *kd, *pe;
    double *x, *u;
    long long* rs;
    int *nup, *node, *status;
    uint32_t* ranks;
    CEOS_D SmemPtrs(unsigned char* raw, const SmemLayout<T>& L)
        : g(reinterpret_cast<T*>(raw + L.g)), ds(reinterpret_cast<T*>(raw + L.ds)),
          st(reinterpret_cast<T*>(raw + L.st)), kd(reinterpret_cast<T*>(raw + L.kd)),
          pe(reinterpret_cast<T*>(raw + L.pe)),
          x(reinterpret_cast<double*>(raw + L.x)), u(reinterpret_cast<double*>(raw + L.u)),
          rs(reinterpret_cast<long long*>(raw + L.rs)),
          nup(reinterpret_cast<int*>(raw + L.nup)), node(reinterpret_cast<int*>(raw + L.node)),
          status(reinterpret_cast<int*>(raw + L.status)), ranks(reinterpret_cast<uint32_t*>(raw + L.ranks)) {}
};

CEOS_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
CEOS_D void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src));
}
CEOS_D void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src));
}
CEOS_D void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src));
}
CEOS_D void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
CEOS_D void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

CEOS_D unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
CEOS_D void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

CEOS_D unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}

// One warp waits until flags[lo..hi) all equal epoch.  Gives up when kWaitNs pass or when another
// CTA has given up (*err set): then it sets *err and returns false.  The result is the same in
// every lane.
CEOS_D bool warp_wait_flags(const unsigned* flags, int lo, int hi, unsigned epoch, int lane, int* err) {
    bool ok = true;
    const unsigned long long t0 = global_ns();
    for (int i = lo + lane; i < hi && ok; i += 32) {
        while (ld_acquire_u32(flags + i) != epoch) {
            if (*reinterpret_cast<volatile int*>(err) != 0 || global_ns() - t0 > kWaitNs) {
                ok = false;
                break;
            }
            __nanosleep(100);
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) atomicOr(err, 1);
    return ok;
}

// Gauss-point state access: committed values from the prefetched shared copy, new values
// streamed to global memory with the evict-first hint (L2 is kept for the K scatter).
template <typename T>
struct StateIO {
    const T* sm;    // &st[0][gp][el]
    T* new_;
    size_t ld8;     // 8 * ld (row stride of one state variable)
    size_t off;     // gp * ld + e
    CEOS_D T ld(int v) const { return sm[v * 8 * kTileE]; }
    CEOS_D void st(int v, T x) const { __stcs(new_ + (size_t)v * ld8 + off, x); }
};

template <typename T, int MODEL>
CEOS_D int run_material(const T F[3][3], const T* p, const T* ebr, double dt, const StateIO<T>& io, T sig[6],
                        T D[21]) {
    constexpr int NS = ModelInfo<MODEL>::nstate;
    int status = 0;
    if constexpr (MODEL == M_CNH) {
        cnh_update<T>(F, p, sig, D);
    } else if constexpr (MODEL == M_SVK) {
        svk_update<T>(F, p, sig, D);
    } else if constexpr (MODEL == M_VISCO_PRONY) {
        visco_prony_update<T>(F, p, ebr, io, sig, D);
    } else if constexpr (MODEL == M_EXTERNAL) {
#pragma unroll
        for (int k = 0; k < 6; ++k) sig[k] = io.ld(k);
#pragma unroll
        for (int k = 0; k < 21; ++k) D[k] = io.ld(6 + k);
    } else {
        T st[NS], stn[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) st[k] = io.ld(k);
        if constexpr (MODEL == M_J2_SMALL) j2_small_update<T>(F, p, st, stn, sig, D);
        else if constexpr (MODEL == M_J2_FINITE) j2_finite_update<T>(F, p, st, stn, sig, D);
        else if constexpr (MODEL == M_VISCO_VAR) status = vv::update<T>(F, p, dt, st, stn, sig, D);
#pragma unroll
        for (int k = 0; k < NS; ++k) io.st(k, stn[k]);
    }
    return status;
}

template <typename T>
CEOS_D void st4(T* p, T a, T b, T c, T d) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
    } else {
        *reinterpret_cast<double2*>(p) = make_double2(a, b);
        *reinterpret_cast<double2*>(p + 2) = make_double2(c, d);
    }
}
template <typename T>
CEOS_D void ld4(const T* p, T& a, T& b, T& c, T& d) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        a = v.x; b = v.y; c = v.z; d = v.w;
    } else {
        const double2 v0 = *reinterpret_cast<const double2*>(p);
        const double2 v1 = *reinterpret_cast<const double2*>(p + 2);
        a = v0.x; b = v0.y; c = v1.x; d = v1.y;
    }
}

// Stage the connectivity and slot ranks of the tile starting at element e0 into one buffer (async).
template <typename T>
CEOS_D void prefetch_conn(const ElemArgs<T>& a, int e0, int* node_s, uint32_t* ranks_s, int t) {
    const int e = t >> 3, n = t & 7;
    if (e0 + e < a.e_end) {
        cp_async4(node_s + n * kTileE + e, a.conn + (size_t)(e0 + e) * 8 + n);
        cp_async4(ranks_s + e * 8 + n, a.ranks + (size_t)(e0 + e) * 8 + n);
    }
}

// Gather node data (X, U, CSR row start, upper-neighbour count) and the committed state of a
// tile whose node ids are already in node_s (async).
template <typename T>
CEOS_D void prefetch_nodes_state(const ElemArgs<T>& a, int e0, const int* node_s, double* xs, double* us,
                                 long long* rs_s, int* nup_s, T* st_s, int t, T* pe_s) {
    const int lane = t & 31, n = t >> 5;
    if (e0 + lane < a.e_end) {
        const int node = node_s[n * kTileE + lane];
        const double* Up = a.U + 3 * (size_t)node;
        double* ud = us + (n * kTileE + lane) * 3;
        {
            const double* Xp = a.X + 3 * (size_t)node;
            double* xd = xs + (n * kTileE + lane) * 3;
#pragma unroll
            for (int d = 0; d < 3; ++d) cp_async8(xd + d, Xp + d);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) cp_async8(ud + d, Up + d);
        cp_async8(rs_s + n * kTileE + lane, a.rs + node);
        cp_async4(nup_s + n * kTileE + lane, a.nup + node);
    }
    if (a.ns_used > 0) {
        constexpr int per_chunk = 16 / sizeof(T);      // elements per 16-byte chunk
        constexpr int cpr = kTileE / per_chunk;        // chunks per (v, gp) row
        const int total = a.ns_used * 8 * cpr;
        for (int c = t; c < total; c += kThreads) {
            const int row = c / cpr, part = c - row * cpr;   // row = v*8 + gp
            cp_async16(st_s + row * kTileE + part * per_chunk, a.st_old + (size_t)row * a.ld + e0 + part * per_chunk);
        }
    }
    // per-element parameters [k][e] (rows of params[k * n_elem + e], not 16-byte aligned in general)
    for (int c = t; c < a.n_pe * kTileE; c += kThreads) {
        const int k = c / kTileE, el = c - k * kTileE;
        if (e0 + el < a.e_end) {
            if constexpr (sizeof(T) == 4) cp_async4(pe_s + c, a.params + (size_t)k * a.n_elem + e0 + el);
            else cp_async8(pe_s + c, a.params + (size_t)k * a.n_elem + e0 + el);
        }
    }
}

CEOS_D void red_v4(float* p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}
CEOS_D void red_v2(float* p, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};\n" ::"l"(p), "f"(a), "f"(b) : "memory");
}

// FP32 mode: node n of element el as differences to the element's node 0, formed in FP64 from the
// staged node data and then rounded: X_n - X_0 and u_n - u_0 keep their relative precision at the
// element scale (absolute coordinates rounded to FP32 would perturb an element of size h by
// ~6e-8 / h, which the bulk modulus of a nearly incompressible material amplifies in f_int).  J_X and
// J_u are unchanged by the shift because sum_n dN_n/dxi = 0.  Each Gauss-point thread forms the
// differences it reads, so the staging needs no conversion pass and no barrier.
CEOS_D void local_node_f32(const SmemPtrs<float>& s, int n, int el, float X[3], float u[3]) {
    const double* xp = s.x + (n * kTileE + el) * 3;
    const double* up = s.u + (n * kTileE + el) * 3;
    const double* x0 = s.x + el * 3;
    const double* u0 = s.u + el * 3;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        X[d] = n == 0 ? 0.f : (float)(xp[d] - x0[d]);
        u[d] = n == 0 ? 0.f : (float)(up[d] - u0[d]);
    }
}

// FP32 mode: the displacement of node n of element el relative to the element's node 0, formed in
// FP64 (J_u is unchanged by the shift because sum_n dN_n/dxi = 0).
CEOS_D void local_u_f32(const SmemPtrs<float>& s, int n, int el, float u[3]) {
    const double* up = s.u + (n * kTileE + el) * 3;
    const double* u0 = s.u + el * 3;
#pragma unroll
    for (int d = 0; d < 3; ++d) u[d] = n == 0 ? 0.f : (float)(up[d] - u0[d]);
}

// Phase A for thread (gp = warp, element = lane) of the tile at e0.
template <typename T, int MODEL>
CEOS_D void phase_a(const ElemArgs<T>& a, const SmemPtrs<T>& s, int e0, int warp, int lane) {
    constexpr int NP = ModelInfo<MODEL>::nparams;
    const int gp = warp, el = lane, e = e0 + el;
    if (e >= a.e_end) return;
    int status = 0;
    // J_X = sum dN/dxi (x) X and J_u = sum dN/dxi (x) u; the current Jacobian is J_X + J_u, and
    // F = I + (J_X^-1 J_u)^T equals DeformationGradient's I + sum u (x) grad_X N with the
    // displacement gradient formed from small numbers (no I + O(1) cancellation in FP32)
    T F[3][3], Jci[3][3], detJ;
    if constexpr (sizeof(T) == 4) {
        // J_X^-1 and det J_X of the reference configuration, computed once per mesh in FP64 on the
        // host ([k][gp][e] rows like the state); J_X + J_u = J_X F^T, so (J_X + J_u)^-1 = F^-T J_X^-1
        // and det = det J_X det F
        const float* q = a.jxi + (size_t)gp * a.ld + e;
        const size_t rstride = (size_t)8 * a.ld;
        float JXi[3][3];
#pragma unroll
        for (int k = 0; k < 9; ++k) JXi[k / 3][k % 3] = __ldg(q + k * rstride);
        const float detJX = __ldg(q + 9 * rstride);
        float Ju[3][3] = {};
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            float u[3];
            local_u_f32(s, n, el, u);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float dn = dN_at<float>(gp, n, i);
#pragma unroll
                for (int j = 0; j < 3; ++j) Ju[i][j] += dn * u[j];
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                F[i][j] = (i == j ? 1.f : 0.f) + (JXi[j][0] * Ju[0][i] + JXi[j][1] * Ju[1][i] + JXi[j][2] * Ju[2][i]);
        const float detF = det3(F);
        detJ = detJX * detF;
        if (!(detJX > 1.0e-13f) || !(detJ > 1.0e-13f)) status |= 1;
        float Fi[3][3];
        inv3(F, detF, Fi);
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) Jci[j][i] = Fi[0][j] * JXi[0][i] + Fi[1][j] * JXi[1][i] + Fi[2][j] * JXi[2][i];
    } else {
        T JX[3][3] = {}, Ju[3][3] = {};
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const double* xp = s.x + (n * kTileE + el) * 3;
            const double* up = s.u + (n * kTileE + el) * 3;
            T X[3], u[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                X[d] = (T)xp[d];
                u[d] = (T)up[d];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T dn = dN_at<T>(gp, n, i);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    JX[i][j] += dn * X[j];
                    Ju[i][j] += dn * u[j];
                }
            }
        }
        T Jc[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Jc[i][j] = JX[i][j] + Ju[i][j];
        const T detJX = det3(JX);
        detJ = det3(Jc);
        if (!(detJX > T(1.0e-13)) || !(detJ > T(1.0e-13))) status |= 1;
        T JXi[3][3];
        inv3(JX, detJX, JXi);
        inv3(Jc, detJ, Jci);
        // F[i][j] = delta_ij + sum_k JXi[j][k] Ju[k][i]
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                F[i][j] = (i == j ? T(1) : T(0)) + (JXi[j][0] * Ju[0][i] + JXi[j][1] * Ju[1][i] + JXi[j][2] * Ju[2][i]);
    }
    // current gradients grad_x N of the 8 nodes for phase B
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const T d0 = dN_at<T>(gp, n, 0), d1 = dN_at<T>(gp, n, 1), d2 = dN_at<T>(gp, n, 2);
        T gx[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) gx[j] = (status & 1) ? T(0) : Jci[j][0] * d0 + Jci[j][1] * d1 + Jci[j][2] * d2;
        st4<T>(s.g + ((gp * 8 + n) * kTileE + el) * 4, gx[0], gx[1], gx[2], T(0));
    }
    // constitutive update
    T p[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        if (a.param_mode == 0) p[k] = a.pu[k];
        else if (a.param_mode == 1) p[k] = s.pe[k * kTileE + el];  // staged with the tile's state
        else p[k] = a.params[(size_t)__ldg(a.mat_id + e) * a.n_params + k];
    }
    StateIO<T> io{s.st + gp * kTileE + el, a.st_new, (size_t)8 * a.ld, (size_t)gp * a.ld + e};
    T sig[6], D[21];
    if (status & 1) {
        if constexpr (MODEL == M_NH_Q1P0)
            if (gp == 0) s.kd[el] = T(0);
#pragma unroll
        for (int k = 0; k < 6; ++k) sig[k] = T(0);
#pragma unroll
        for (int k = 0; k < 21; ++k) D[k] = T(0);
        for (int k = 0; k < a.ns_used; ++k) io.st(k, io.ld(k));
    } else {
        T ebr[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (MODEL == M_VISCO_PRONY && a.param_mode != 0)
                ebr[k] = texp<T>((T)(-a.dt) / (T(2) * p[4 + 2 * k]));
            else
                ebr[k] = a.ebr[k];
        }
        if constexpr (MODEL == M_NH_Q1P0) {
            // Jbar = V / V0 (ElementVolume, ModElement.f90:1313-1427): every Gauss-point
            // thread of the element sums the same 8 determinants (no barrier needed)
            double V = 0.0, V0 = 0.0;
#pragma unroll 1
            for (int g2 = 0; g2 < 8; ++g2) {
                T JX2[3][3] = {}, Jc2[3][3] = {};
#pragma unroll
                for (int n = 0; n < 8; ++n) {
                    T X[3], x[3];
                    if constexpr (sizeof(T) == 4) {
                        float uf[3];
                        local_node_f32(s, n, el, X, uf);
                        x[0] = X[0] + uf[0]; x[1] = X[1] + uf[1]; x[2] = X[2] + uf[2];
                    } else {
                        const double* xp = s.x + (n * kTileE + el) * 3;
                        const double* up = s.u + (n * kTileE + el) * 3;
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            X[d] = (T)xp[d];
                            x[d] = (T)(xp[d] + up[d]);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const T dn = dN_at<T>(g2, n, i);
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            JX2[i][j] += dn * X[j];
                            Jc2[i][j] += dn * x[j];
                        }
                    }
                }
                V0 += (double)det3(JX2);
                V += (double)det3(Jc2);
            }
            const double Jbar = V / V0;
            nh_q1p0_update<T>(F, p, Jbar, sig, D);
            if (gp == 0) s.kd[el] = (T)(nh_q1p0_d2psi((double)p[1], Jbar) / V0);
        } else {
            status |= run_material<T, MODEL>(F, p, ebr, a.dt, io, sig, D);
        }
    }
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 6; ++k) finite = finite && isfinite(sig[k]);
    if (!finite) status |= 4;
    if (a.gp_stress) {
#pragma unroll
        for (int k = 0; k < 6; ++k) a.gp_stress[((size_t)k * 8 + gp) * a.n_elem + e] = sig[k];
    }
    const T w = (status & 5) ? T(0) : detJ;  // Gauss weight is 1 (Hexa8 full integration)
    T* dst = s.ds + (size_t)gp * 7 * kTileE * 4 + el * 4;
#pragma unroll
    for (int q = 0; q < 5; ++q)
        st4<T>(dst + q * kTileE * 4, w * D[4 * q], w * D[4 * q + 1], w * D[4 * q + 2], w * D[4 * q + 3]);
    st4<T>(dst + 5 * kTileE * 4, w * D[20], w * sig[0], w * sig[1], w * sig[2]);
    st4<T>(dst + 6 * kTileE * 4, w * sig[3], w * sig[4], w * sig[5], w);  // w: Mean Dilatation
    if (status) atomicOr(&s.status[el], status);
}

// Element status of the tile (threads t < kTileE), then clear the shared status words.
template <typename T>
CEOS_D void tile_status(const ElemArgs<T>& a, const SmemPtrs<T>& s, int e0, int t) {
    if (t < kTileE) {
        if (e0 + t < a.e_end) {
            const int st = s.status[t];
            a.elem_status[e0 + t] = (uint8_t)st;
            if (st) atomicAdd(a.status_count, 1);
        }
        s.status[t] = 0;
    }
}

enum : int { SCATTER_CSR64 = 0, SCATTER_RING = 1 };

// Phase B for thread (node b = warp, element = lane) of the tile at e0; node_c, rs_c, nup_c and
// ranks_c are the tile's buffers.  SCATTER_CSR64: K by FP64 atomics into the CSR values (skipped
// when a.kval is null); SCATTER_RING: K by FP32 vector reductions into the node-pair block ring.
template <typename T, int MODEL, int SCATTER>
CEOS_D void phase_b(const ElemArgs<T>& a, const SmemPtrs<T>& s, int e0, int warp, int lane, const int* node_c,
                    const long long* rs_c, const int* nup_c, const uint32_t* ranks_c) {
    const int b = warp, el = lane, e = e0 + el;
    if (e >= a.e_end) return;
    const int npair = (b < 4) ? 4 : 3;  // off-diagonal partners a = b+1..b+npair (mod 8)
    T f0 = 0, f1 = 0, f2 = 0;
    T Kd[6] = {0, 0, 0, 0, 0, 0};
    T Ko[4][9];
    // Mean Dilatation: Bdiv of node b and of its partners, sum_gp w detJ grad N (current)
    T bdb[3] = {T(0), T(0), T(0)}, bda[4][3] = {};
    // FP32: the 3x3 blocks accumulate two columns per packed FMA (sm_100 FFMA2).  Row 0
    // pairs column 2 with the geometric term g_a . sigma g_b, which enters the diagonal
    // of the block once after the Gauss-point loop.
    float2 Pa[4][3], Pc[4], Da = {0.f, 0.f}, Dc = {0.f, 0.f};
    float Pr[4][2], d11 = 0.f, d12 = 0.f, d22 = 0.f;
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            Pa[o][0] = Pa[o][1] = Pa[o][2] = Pc[o] = make_float2(0.f, 0.f);
            Pr[o][0] = Pr[o][1] = 0.f;
        }
    } else {
#pragma unroll
        for (int o = 0; o < 4; ++o)
#pragma unroll
            for (int k = 0; k < 9; ++k) Ko[o][k] = T(0);
    }
#pragma unroll 2
    for (int gp = 0; gp < 8; ++gp) {
        const T* src = s.ds + (size_t)gp * 7 * kTileE * 4 + el * 4;
        T Dm[21], s0, s1, s2, s3, s4, s5, pad;
#pragma unroll
        for (int q = 0; q < 5; ++q)
            ld4<T>(src + q * kTileE * 4, Dm[4 * q], Dm[4 * q + 1], Dm[4 * q + 2], Dm[4 * q + 3]);
        ld4<T>(src + 5 * kTileE * 4, Dm[20], s0, s1, s2);
        T wgp;
        ld4<T>(src + 6 * kTileE * 4, s3, s4, s5, wgp);
        const T* gsrc = s.g + (size_t)gp * 8 * kTileE * 4 + el * 4;
        T gx, gy, gz;
        ld4<T>(gsrc + b * kTileE * 4, gx, gy, gz, pad);
        if constexpr (MODEL == M_NH_Q1P0) {
            bdb[0] += wgp * gx;
            bdb[1] += wgp * gy;
            bdb[2] += wgp * gz;
        }
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
        if constexpr (sizeof(T) == 4) {
            float2 P[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) P[i] = make_float2(DB[i][0], DB[i][1]);
            const float2 z0 = make_float2(DB[0][2], q0), z3 = make_float2(DB[3][2], q1),
                         z5 = make_float2(DB[5][2], q2);
            {   // diagonal block (b,b), upper 6
                const float2 bx = make_float2(gx, gx), by = make_float2(gy, gy), bz = make_float2(gz, gz);
                Da = __ffma2_rn(bx, P[0], Da); Da = __ffma2_rn(by, P[3], Da); Da = __ffma2_rn(bz, P[5], Da);
                Dc = __ffma2_rn(bx, z0, Dc);   Dc = __ffma2_rn(by, z3, Dc);   Dc = __ffma2_rn(bz, z5, Dc);
                d11 += gy * P[1].y + gx * P[3].y + gz * P[4].y;
                d12 += gy * DB[1][2] + gx * DB[3][2] + gz * DB[4][2];
                d22 += gz * DB[2][2] + gy * DB[4][2] + gx * DB[5][2];
            }
#pragma unroll
            for (int o = 0; o < 4; ++o) {
                if (o < npair) {
                    const int an = (b + 1 + o) & 7;
                    T ax, ay, az;
                    ld4<T>(gsrc + an * kTileE * 4, ax, ay, az, pad);
                    if constexpr (MODEL == M_NH_Q1P0) {
                        bda[o][0] += wgp * ax;
                        bda[o][1] += wgp * ay;
                        bda[o][2] += wgp * az;
                    }
                    const float2 bx = make_float2(ax, ax), by = make_float2(ay, ay), bz = make_float2(az, az);
                    Pa[o][0] = __ffma2_rn(bx, P[0], Pa[o][0]);
                    Pa[o][0] = __ffma2_rn(by, P[3], Pa[o][0]);
                    Pa[o][0] = __ffma2_rn(bz, P[5], Pa[o][0]);
                    Pc[o] = __ffma2_rn(bx, z0, Pc[o]);
                    Pc[o] = __ffma2_rn(by, z3, Pc[o]);
                    Pc[o] = __ffma2_rn(bz, z5, Pc[o]);
                    Pa[o][1] = __ffma2_rn(by, P[1], Pa[o][1]);
                    Pa[o][1] = __ffma2_rn(bx, P[3], Pa[o][1]);
                    Pa[o][1] = __ffma2_rn(bz, P[4], Pa[o][1]);
                    Pr[o][0] += ay * DB[1][2] + ax * DB[3][2] + az * DB[4][2];
                    Pa[o][2] = __ffma2_rn(bz, P[2], Pa[o][2]);
                    Pa[o][2] = __ffma2_rn(by, P[4], Pa[o][2]);
                    Pa[o][2] = __ffma2_rn(bx, P[5], Pa[o][2]);
                    Pr[o][1] += az * DB[2][2] + ay * DB[4][2] + ax * DB[5][2];
                }
            }
        } else {
            // diagonal block (b,b), upper 6
            {
                const T geo = gx * q0 + gy * q1 + gz * q2;
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
                    T ax, ay, az;
                    ld4<T>(gsrc + an * kTileE * 4, ax, ay, az, pad);
                    const T geo = ax * q0 + ay * q1 + az * q2;
                    if constexpr (MODEL == M_NH_Q1P0) {
                        bda[o][0] += wgp * ax;
                        bda[o][1] += wgp * ay;
                        bda[o][2] += wgp * az;
                    }
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
    }
    if constexpr (sizeof(T) == 4) {  // unpack the column pairs, add the geometric terms
        const float gb = Dc.y;
        Kd[0] = Da.x + gb; Kd[1] = Da.y; Kd[2] = Dc.x;
        Kd[3] = d11 + gb;  Kd[4] = d12;  Kd[5] = d22 + gb;
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            const float ga = Pc[o].y;
            Ko[o][0] = Pa[o][0].x + ga; Ko[o][1] = Pa[o][0].y; Ko[o][2] = Pc[o].x;
            Ko[o][3] = Pa[o][1].x;      Ko[o][4] = Pa[o][1].y + ga; Ko[o][5] = Pr[o][0];
            Ko[o][6] = Pa[o][2].x;      Ko[o][7] = Pa[o][2].y; Ko[o][8] = Pr[o][1] + ga;
        }
    }
    if constexpr (MODEL == M_NH_Q1P0) {  // Bdiv^T Bdiv d2psi/dJbar2 / V0 (ModElement.f90:463-466)
        const T kd = isfinite(s.kd[el]) ? s.kd[el] : T(0);  // failed elements have Bdiv = 0
        Kd[0] += kd * bdb[0] * bdb[0];
        Kd[1] += kd * bdb[0] * bdb[1];
        Kd[2] += kd * bdb[0] * bdb[2];
        Kd[3] += kd * bdb[1] * bdb[1];
        Kd[4] += kd * bdb[1] * bdb[2];
        Kd[5] += kd * bdb[2] * bdb[2];
#pragma unroll
        for (int o = 0; o < 4; ++o)
            if (o < npair)
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int l = 0; l < 3; ++l) Ko[o][k * 3 + l] += kd * bda[o][k] * bdb[l];
    }
    // ---- scatter ----
    const int Bn = node_c[b * kTileE + el];
    atomicAdd(a.fint + 3 * (size_t)Bn + 0, (double)f0);
    atomicAdd(a.fint + 3 * (size_t)Bn + 1, (double)f1);
    atomicAdd(a.fint + 3 * (size_t)Bn + 2, (double)f2);
    if constexpr (SCATTER == SCATTER_CSR64) {
        if (!a.kval) return;
        {
            const long long r0 = rs_c[b * kTileE + el];
            const int m = nup_c[b * kTileE + el];
            const long long r1 = r0 + 3 + 3 * m, r2 = r1 + 2 + 3 * m;
            double* K = a.kval;
            atomicAdd(K + r0 + 0, (double)Kd[0]);
            atomicAdd(K + r0 + 1, (double)Kd[1]);
            atomicAdd(K + r0 + 2, (double)Kd[2]);
            atomicAdd(K + r1 + 0, (double)Kd[3]);
            atomicAdd(K + r1 + 1, (double)Kd[4]);
            atomicAdd(K + r2 + 0, (double)Kd[5]);
        }
        const uint8_t* rk = reinterpret_cast<const uint8_t*>(ranks_c + el * 8);
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            if (o < npair) {
                const int an = (b + 1 + o) & 7;
                const int An = node_c[an * kTileE + el];
                const int lo_local = an < b ? an : b, hi_local = an < b ? b : an;
                const int r = rk[pair_index(lo_local, hi_local)];
                const bool a_low = An < Bn;  // rows belong to the smaller global node
                const int lo_n = a_low ? an : b;
                const long long r0 = rs_c[lo_n * kTileE + el];
                const int m = nup_c[lo_n * kTileE + el];
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
    } else {
        // node-pair blocks in the ring: one 16-byte vector reduction per block row; rs_c holds the
        // first block of each node, the slot of block q is q & ring_mask
        const uint32_t mask = a.ring_mask;
        {
            float* blk = a.kblk + (size_t)((uint32_t)rs_c[b * kTileE + el] & mask) * 12;
            // diagonal block: its upper 6 entries packed as K00 K01 K02 K11 | K12 K22 (two reductions)
            red_v4(blk + 0, (float)Kd[0], (float)Kd[1], (float)Kd[2], (float)Kd[3]);
            red_v2(blk + 4, (float)Kd[4], (float)Kd[5]);
        }
        const uint8_t* rk = reinterpret_cast<const uint8_t*>(ranks_c + el * 8);
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            if (o < npair) {
                const int an = (b + 1 + o) & 7;
                const int An = node_c[an * kTileE + el];
                const int lo_local = an < b ? an : b, hi_local = an < b ? b : an;
                const int r = rk[pair_index(lo_local, hi_local)];
                const bool a_low = An < Bn;
                const int lo_n = a_low ? an : b;
                float* blk = a.kblk + (size_t)(((uint32_t)rs_c[lo_n * kTileE + el] + 1u + (uint32_t)r) & mask) * 12;
                if (a_low) {  // rows of node a: M[k][:]
                    red_v4(blk + 0, (float)Ko[o][0], (float)Ko[o][1], (float)Ko[o][2], 0.f);
                    red_v4(blk + 4, (float)Ko[o][3], (float)Ko[o][4], (float)Ko[o][5], 0.f);
                    red_v4(blk + 8, (float)Ko[o][6], (float)Ko[o][7], (float)Ko[o][8], 0.f);
                } else {      // rows of node b: M[:][l]
                    red_v4(blk + 0, (float)Ko[o][0], (float)Ko[o][3], (float)Ko[o][6], 0.f);
                    red_v4(blk + 4, (float)Ko[o][1], (float)Ko[o][4], (float)Ko[o][7], 0.f);
                    red_v4(blk + 8, (float)Ko[o][2], (float)Ko[o][5], (float)Ko[o][8], 0.f);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Static schedule: FP64 mode (K by FP64 atomics), evaluations without a tangent, and the element
// pass of the two-pass mixed-precision assembly (K blocks into the scratch, SCATTER_RING)
// ---------------------------------------------------------------------------------------------
template <typename T, int MODEL, int SCATTER = SCATTER_CSR64>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1) element_loop_kernel(ElemArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemLayout<T> L(a.ns_used, a.n_pe);
    const SmemPtrs<T> s(smem_raw, L);
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int n_tiles = (a.e_end - a.e_begin + kTileE - 1) / kTileE;
    constexpr int NB = 8 * kTileE;  // one buffer of [node][e] ints

    int tile = blockIdx.x;
    if (tile >= n_tiles) return;
    // prologue: connectivity of the first tile, then its node data and state
    prefetch_conn(a, a.e_begin + tile * kTileE, s.node, s.ranks, t);
    cp_commit();
    if (t < kTileE) s.status[t] = 0;
    cp_wait_all();
    __syncthreads();
    prefetch_nodes_state(a, a.e_begin + tile * kTileE, s.node, s.x, s.u, s.rs, s.nup, s.st, t, s.pe);
    cp_commit();

    for (int it = 0; tile < n_tiles; ++it, tile += gridDim.x) {
        const int buf = it & 1;
        const int e0 = a.e_begin + tile * kTileE;
        const int next = tile + gridDim.x;
        const int e0n = a.e_begin + next * kTileE;
        cp_wait_all();
        __syncthreads();  // node data and state of this tile are in shared memory
        if (next < n_tiles) {
            prefetch_conn(a, e0n, s.node + (buf ^ 1) * NB, s.ranks + (buf ^ 1) * NB, t);
            cp_commit();
        }
        phase_a<T, MODEL>(a, s, e0, warp, lane);
        cp_wait_all();    // connectivity of the next tile has landed
        __syncthreads();  // phase A results visible; x, u and state buffers are free
        if (next < n_tiles) {
            prefetch_nodes_state(a, e0n, s.node + (buf ^ 1) * NB, s.x, s.u, s.rs + (buf ^ 1) * NB,
                                 s.nup + (buf ^ 1) * NB, s.st, t, s.pe);
            cp_commit();
        }
        tile_status(a, s, e0, t);
        phase_b<T, MODEL, SCATTER>(a, s, e0, warp, lane, s.node + buf * NB, s.rs + buf * NB, s.nup + buf * NB,
                                   s.ranks + buf * NB);
    }
    cp_wait_all();
}

// ---------------------------------------------------------------------------------------------
// Fused schedule (CEOS_MIXED with a tangent): element tiles and CSR conversion items
// ---------------------------------------------------------------------------------------------

// Conversion item: the CSR rows of nodes [n0, n1) (at most kConvNodes) from their ring blocks.
// The blocks of consecutive nodes are consecutive, [blk0[n0], blk0[n1-1] + 1 + nup[n1-1]), and so
// are their K values, from csr_rs[n0].  A table of the item's nodes is read first (one load per
// node); then every thread takes whole blocks and issues the loads of all three rows of its blocks
// before it uses any, so that an item costs a few memory latencies rather than one per node.  The
// FP64 values are staged in shared memory and the K run is written with 16-byte streaming stores;
// the ring blocks are re-zeroed for their next occupant.
template <int kU>  // blocks in flight per thread
CEOS_D void convert_rows(const ElemArgs<float>& a, int n0, int n1, double* stage, int* info, int t) {
    int* fb = info;                   // first block of the node, relative to the item's first block
    int* fk = info + kConvNodes;      // stage index of the node's first K value
    int* fm = info + 2 * kConvNodes;  // upper neighbours of the node
    const long long base = __ldg(a.csr_rs + n0);
    const int head = (int)(base & 1);  // stage index of K[base + p] is p + head (16-byte pairs)
    const uint32_t b0 = (uint32_t)__ldg(a.rs + n0);
    const int nn = n1 - n0;
    for (int i = t; i < nn; i += kThreads) {
        fb[i] = (int)((uint32_t)__ldg(a.rs + n0 + i) - b0);
        fk[i] = (int)(__ldg(a.csr_rs + n0 + i) - base) + head;
        fm[i] = __ldg(a.nup + n0 + i);
    }
    __syncthreads();
    const int nblk = fb[nn - 1] + 1 + fm[nn - 1];
    const uint32_t mask = a.ring_mask;
    for (int q0 = t; q0 < nblk; q0 += kU * kThreads) {
        float4 v[kU][3];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int q = q0 + u * kThreads;
            if (q < nblk) {
                const float4* src = reinterpret_cast<const float4*>(a.kblk + (size_t)((b0 + (uint32_t)q) & mask) * 12);
#pragma unroll
                for (int k = 0; k < 3; ++k) v[u][k] = __ldcg(src + k);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int q = q0 + u * kThreads;
            if (q >= nblk) continue;
            float4* src = reinterpret_cast<float4*>(a.kblk + (size_t)((b0 + (uint32_t)q) & mask) * 12);
#pragma unroll
            for (int k = 0; k < 3; ++k) __stcg(src + k, make_float4(0.f, 0.f, 0.f, 0.f));
            int lo = 0, hi = nn - 1;  // the node of block q: the last i with fb[i] <= q
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (fb[mid] <= q) lo = mid;
                else hi = mid - 1;
            }
            const int j = q - fb[lo], m = fm[lo], rel = fk[lo];
            const int r1 = rel + 3 + 3 * m, r2 = r1 + 2 + 3 * m;  // rows 3n+1 and 3n+2
            if (j == 0) {  // diagonal block, packed: K00 K01 K02 K11 | K12 K22
                stage[rel] = v[u][0].x; stage[rel + 1] = v[u][0].y; stage[rel + 2] = v[u][0].z;
                stage[r1] = v[u][0].w; stage[r1 + 1] = v[u][1].x;
                stage[r2] = v[u][1].y;
            } else {
                double* d0 = stage + rel + 3 + 3 * (j - 1);
                double* d1 = stage + r1 + 2 + 3 * (j - 1);
                double* d2 = stage + r2 + 1 + 3 * (j - 1);
                d0[0] = v[u][0].x; d0[1] = v[u][0].y; d0[2] = v[u][0].z;
                d1[0] = v[u][1].x; d1[1] = v[u][1].y; d1[2] = v[u][1].z;
                d2[0] = v[u][2].x; d2[1] = v[u][2].y; d2[2] = v[u][2].z;
            }
        }
    }
    __syncthreads();
    const int L = fk[nn - 1] - head + 6 + 9 * fm[nn - 1];
    double* K = a.kval + base - head;  // 16-byte aligned: base - head is even
    const int npairs = (L + head + 1) >> 1;
    for (int i = t; i < npairs; i += kThreads) {
        const int p0 = 2 * i, p1 = p0 + 1;
        if (p0 >= head && p1 < head + L) {
            __stcs(reinterpret_cast<double2*>(K + p0), *reinterpret_cast<const double2*>(stage + p0));
        } else {
            if (p0 >= head && p0 < head + L) __stcs(K + p0, stage[p0]);
            if (p1 >= head && p1 < head + L) __stcs(K + p1, stage[p1]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Conversion pass of the two-pass and banded assemblies (csr_convert_kernel)
// ---------------------------------------------------------------------------------------------
// Items of this pass hold at most kBulkNodes nodes and kBulkStage - 1 K values, so at most
// kBulkBlocks node-pair blocks (blocks = nodes + sum of upper neighbours <= nodes + values / 9).
// Shared memory: two block buffers | FP64 staging of one item | node table | two mbarriers.
constexpr int kBulkNodes = 96;
constexpr int kBulkStage = 2048;
constexpr int kBulkBlocks = kBulkNodes + kBulkStage / 9 + 1;
constexpr int kBulkRawBytes = kBulkBlocks * 48;
constexpr int kBulkStageOff = 2 * kBulkRawBytes;
constexpr int kBulkTableOff = kBulkStageOff + (kBulkStage + 2) * 8;
constexpr int kBulkMbarOff = kBulkTableOff + 3 * kBulkNodes * 4;
constexpr int kBulkSmem = kBulkMbarOff + 16;
static_assert(kBulkRawBytes % 16 == 0 && kBulkStageOff % 16 == 0 && kBulkMbarOff % 8 == 0, "bulk copy alignment");
static_assert(kBulkStage <= kStageDoubles && kBulkNodes <= kConvNodes, "items must also fit the fused staging");

CEOS_D void mbar_init(uint64_t* m) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(m)) : "memory");
}
CEOS_D void mbar_expect_tx(uint64_t* m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
CEOS_D bool mbar_try_wait(uint64_t* m, unsigned parity) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(done) : "r"(smem_u32(m)), "r"(parity) : "memory");
    return done != 0;
}
// Waits for phase `parity` of m for at most kWaitNs; false when the bound ran out.
CEOS_D bool mbar_wait_bounded(uint64_t* m, unsigned parity) {
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(m, parity))
        if (global_ns() - t0 > kWaitNs) return false;
    return true;
}
// global -> shared bulk copy (no multicast) completing on mbarrier m; 16-byte aligned, size % 16 == 0
CEOS_D void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m)) : "memory");
}
// shared -> global bulk copy in the thread's bulk group; 16-byte aligned, size % 16 == 0
CEOS_D void bulk_store(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n"
                 ::"l"(dst), "r"(smem_u32(src)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
CEOS_D void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
CEOS_D void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
CEOS_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Node table of an item, loaded one item ahead into registers: thread t < nodes holds node n0 + t.
struct ConvRow {
    long long blk, pos;  // first node-pair block and first K position of the node
    int up;              // upper neighbours
};

// CTA k converts the items order[j0 + k], order[j0 + k + gridDim.x], ... < j1 (the conversion items of
// one element slab, or all of them; items j themselves when order is null, as for the bands of the
// banded assembly); the element passes before it in stream order have completed every reduction
// into their blocks.  Software pipeline over the CTA's items, one item ahead:
//   thread 0 fetches the next item's blocks (one contiguous run of 48-byte blocks, two runs where
//   it wraps around the ring) into the other block buffer with bulk copies on an mbarrier, from the
//   item's host-built metadata (no dependent loads);
//   every thread keeps the next item's node table in registers while it converts the current one,
//   waits for the current item's blocks, turns whole blocks into the FP64 staging (the node of a
//   block by binary search in the table) and re-zeroes them in HBM;
//   thread 0 writes the item's contiguous K run with one bulk store (16-byte aligned middle; the
//   odd first and last values by plain stores), which drains while the next item converts.
// Every wait is bounded: a copy that does not land within kWaitNs sets *sched_err (reported as
// CEOS_E_CUDA, and the next evaluation clears the blocks) and the CTA stops after waiting, again
// bounded, for the copies it still has in flight.
__global__ void __launch_bounds__(kThreads, 4) csr_convert_kernel(ElemArgs<float> a, const int* order, int j0, int j1) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* raw0 = reinterpret_cast<float*>(smem_raw);
    float* raw1 = reinterpret_cast<float*>(smem_raw + kBulkRawBytes);
    double* stage = reinterpret_cast<double*>(smem_raw + kBulkStageOff);
    int* fb = reinterpret_cast<int*>(smem_raw + kBulkTableOff);  // first block, relative to the item's
    int* fk = fb + kBulkNodes;                                    // stage index of the first K value
    int* fm = fk + kBulkNodes;                                    // upper neighbours
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + kBulkMbarOff);
    __shared__ int s_fail;
    __shared__ int s_issued[2];
    const int t = threadIdx.x;
    const int g = (int)gridDim.x;
    int j = j0 + (int)blockIdx.x;
    if (j >= j1) return;
    const unsigned long long mask = a.ring_mask, ring = mask + 1ull;
    struct Meta {
        long long b0, base;
        int n0, nn, nblk, nval;
    };
    auto meta = [&](int jj) {
        const int id = order ? __ldg(order + jj) : jj;
        const longlong2 p = __ldg(a.conv_meta + 2 * (size_t)id), q = __ldg(a.conv_meta + 2 * (size_t)id + 1);
        return Meta{p.x, p.y, (int)(q.x & 0xffffffffLL), (int)(q.x >> 32), (int)(q.y & 0xffffffffLL), (int)(q.y >> 32)};
    };
    auto row = [&](const Meta& m) {
        ConvRow r{0, 0, 0};
        if (t < m.nn && m.nn <= kBulkNodes) {
            r.blk = __ldg(a.rs + m.n0 + t);
            r.pos = __ldg(a.csr_rs + m.n0 + t);
            r.up = __ldg(a.nup + m.n0 + t);
        }
        return r;
    };
    auto in_bounds = [](const Meta& m) {
        return m.nn >= 1 && m.nn <= kBulkNodes && m.nblk >= 1 && m.nblk <= kBulkBlocks && m.nval >= 6 &&
               m.nval <= kBulkStage - 1;
    };
    // thread 0: bulk copies of the blocks of an item into buffer bf
    auto issue = [&](const Meta& m, int bf) {
        if (!in_bounds(m)) {
            s_issued[bf] = 0;  // outside the planned bounds (the host checks them): never happens
            return;
        }
        float* dst = bf ? raw1 : raw0;
        mbar_expect_tx(mbar + bf, (unsigned)m.nblk * 48u);
        const unsigned long long s0 = (unsigned long long)m.b0 & mask;
        const unsigned long long na = (unsigned long long)m.nblk < ring - s0 ? (unsigned long long)m.nblk : ring - s0;
        bulk_load(dst, a.kblk + s0 * 12, (unsigned)na * 48u, mbar + bf);
        if (na < (unsigned long long)m.nblk) bulk_load(dst + na * 12, a.kblk, (unsigned)(m.nblk - (int)na) * 48u, mbar + bf);
        s_issued[bf] = 1;
    };
    unsigned ph0 = 0, ph1 = 0;  // parity of the next phase of each buffer's mbarrier
    int pend0 = 0, pend1 = 0;   // loads issued into each buffer and not yet landed (used by thread 0)
    Meta mc = meta(j);                                   // current item
    ConvRow rc = row(mc);                                // its node table
    Meta mn = j + g < j1 ? meta(j + g) : Meta{0, 0, 0, 0, 0, 0};  // next item
    if (t == 0) {
        mbar_init(mbar);
        mbar_init(mbar + 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_fail = 0;
        issue(mc, 0);
        pend0 = s_issued[0];
    }
    __syncthreads();
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; j < j1; ++k, j += g) {
        const int buf = k & 1;
        const bool has_next = j + g < j1;
        if (t == 0 && has_next) {  // the other buffer was last read before the end of the previous item
            fence_proxy_async();
            issue(mn, buf ^ 1);
            if (buf) pend0 = s_issued[0];
            else pend1 = s_issued[1];
        }
        // the current item's table into shared memory (the previous item stopped reading it before
        // the end of its conversion); the next item's table and the one after's metadata are loaded
        // now and used one item later
        const int head = (int)(mc.base & 1);  // stage index of K[base + p] is p + head (16-byte pairs)
        if (t < mc.nn && mc.nn <= kBulkNodes) {
            fb[t] = (int)(rc.blk - mc.b0);
            fk[t] = (int)(rc.pos - mc.base) + head;
            fm[t] = rc.up;
        }
        const ConvRow rn = has_next ? row(mn) : ConvRow{0, 0, 0};
        const Meta mnn = j + 2 * g < j1 ? meta(j + 2 * g) : Meta{0, 0, 0, 0, 0, 0};
        if (s_issued[buf]) {
            // the phase of a load that did not land stays current: the clean-up waits for it again
            if (mbar_wait_bounded(mbar + buf, buf ? ph1 : ph0)) {
                if (buf) {
                    ph1 ^= 1u;
                    pend1 = 0;
                } else {
                    ph0 ^= 1u;
                    pend0 = 0;
                }
            } else {
                atomicOr(&s_fail, 1);
            }
        } else if (t == 0) {
            atomicOr(&s_fail, 2);
        }
        if (t == 0) bulk_wait_read_all();  // the previous item's K store has read the staging
        __syncthreads();
        if (s_fail) break;
        const float* rb = buf ? raw1 : raw0;
        const int nn = mc.nn, nblk = mc.nblk, L = mc.nval;
        for (int q = t; q < nblk; q += kThreads) {
            const float4* src = reinterpret_cast<const float4*>(rb + (size_t)q * 12);
            const float4 v0 = src[0], v1 = src[1], v2 = src[2];
            float4* gb = reinterpret_cast<float4*>(a.kblk + (size_t)(((unsigned long long)mc.b0 + q) & mask) * 12);
            __stcg(gb, zero);  // re-zero the slot for the next evaluation
            __stcg(gb + 1, zero);
            __stcg(gb + 2, zero);
            int lo = 0, hi = nn - 1;  // the node of block q: the last i with fb[i] <= q
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (fb[mid] <= q) lo = mid;
                else hi = mid - 1;
            }
            const int jb = q - fb[lo], m = fm[lo], rel = fk[lo];
            const int r1 = rel + 3 + 3 * m, r2 = r1 + 2 + 3 * m;  // rows 3n+1 and 3n+2
            if (jb == 0) {  // diagonal block, packed: K00 K01 K02 K11 | K12 K22
                stage[rel] = v0.x; stage[rel + 1] = v0.y; stage[rel + 2] = v0.z;
                stage[r1] = v0.w; stage[r1 + 1] = v1.x;
                stage[r2] = v1.y;
            } else {
                double* d0 = stage + rel + 3 + 3 * (jb - 1);
                double* d1 = stage + r1 + 2 + 3 * (jb - 1);
                double* d2 = stage + r2 + 1 + 3 * (jb - 1);
                d0[0] = v0.x; d0[1] = v0.y; d0[2] = v0.z;
                d1[0] = v1.x; d1[1] = v1.y; d1[2] = v1.z;
                d2[0] = v2.x; d2[1] = v2.y; d2[2] = v2.z;
            }
        }
        fence_proxy_async();  // staging writes (and block reads) ordered before the bulk copies that follow
        __syncthreads();
        double* K = a.kval + mc.base - head;  // 16-byte aligned: base - head is even
        const int pa = (head + 1) & ~1, pb = (head + L) & ~1;
        if (pb > pa) {
            if (t == 0) bulk_store(K + pa, stage + pa, (unsigned)(pb - pa) * 8u);
            if (t == 32 && head) __stcs(K + 1, stage[1]);
            if (t == 64 && ((head + L) & 1)) __stcs(K + head + L - 1, stage[head + L - 1]);
        } else {
            for (int p = head + t; p < head + L; p += kThreads) __stcs(K + p, stage[p]);
        }
        mc = mn;
        rc = rn;
        mn = mnn;
    }
    if (t == 0) {
        if (s_fail) {
            if (a.sched_err) atomicOr(a.sched_err, 1);
            // copies still in flight into this CTA's shared memory: wait for them, bounded
            if (pend0) (void)mbar_wait_bounded(mbar, ph0);
            if (pend1) (void)mbar_wait_bounded(mbar + 1, ph1);
        }
        bulk_wait_all();  // the K stores are complete
    }
}

template <int MODEL>
__global__ void __launch_bounds__(kThreads, 2) element_assemble_kernel(ElemArgs<float> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item[2];
    __shared__ int s_abort;
    const SmemLayout<float> L(a.ns_used, a.n_pe);
    const SmemPtrs<float> s(smem_raw, L);
    double* stage = reinterpret_cast<double*>(smem_raw + L.g);  // g and ds are contiguous
    int* conv_info = reinterpret_cast<int*>(stage + kStageDoubles + 2);
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    constexpr int NB = 8 * kTileE;

    auto item_at = [&](unsigned k) -> int {
        const long long pos = (long long)a.q_begin + k;
        return pos < a.q_end ? __ldg(a.queue + pos) : kEndItem;
    };
    // Tickets run one item ahead of use: while an item is processed, the ticket after the next one is
    // already requested, so the atomic's latency is hidden behind the work.  A CTA holds at most three
    // tickets (current, next, requested); each waits only for earlier queue positions.
    int slot = 0;
    if (t == 0) {
        s_item[0] = item_at(atomicAdd(a.ticket, 1u));
        s_item[1] = item_at(atomicAdd(a.ticket, 1u));
        s_abort = 0;
    }
    if (t < kTileE) s.status[t] = 0;
    __syncthreads();
    int cur = s_item[0];
    int next = s_item[1];
    int buf = 0;  // the connectivity and node data of `cur` (a tile) are staged in buffer buf
    if (cur >= 0) {
        prefetch_conn(a, cur * kTileE, s.node, s.ranks, t);
        cp_commit();
        cp_wait_all();
        __syncthreads();
        prefetch_nodes_state(a, cur * kTileE, s.node, s.x, s.u, s.rs, s.nup, s.st, t, s.pe);
        cp_commit();
    }
    while (cur != kEndItem) {
        unsigned requested = 0;
        if (t == 0) requested = atomicAdd(a.ticket, 1u);
        if (cur >= 0) {
            // ---------------- element tile ----------------
            const int e0 = cur * kTileE;
            const int nb = buf ^ 1;
            cp_wait_all();
            __syncthreads();  // node data and state of this tile are in shared memory
            if (next >= 0) {
                prefetch_conn(a, next * kTileE, s.node + nb * NB, s.ranks + nb * NB, t);
                cp_commit();
            }
            phase_a<float, MODEL>(a, s, e0, warp, lane);
            if (warp == 0) {  // the ring slots of this tile must have been released by their last user
                const int2 wr = __ldg(a.tile_wait + cur);
                if (wr.y > wr.x && !warp_wait_flags(a.conv_done, wr.x, wr.y, a.epoch, lane, a.sched_err) && lane == 0)
                    s_abort = 1;
            }
            cp_wait_all();    // connectivity of the next tile has landed
            __syncthreads();  // phase A results visible; x, u and state buffers are free
            if (s_abort) break;
            if (next >= 0) {
                prefetch_nodes_state(a, next * kTileE, s.node + nb * NB, s.x, s.u, s.rs + nb * NB, s.nup + nb * NB,
                                     s.st, t, s.pe);
                cp_commit();
            }
            tile_status(a, s, e0, t);
            phase_b<float, MODEL, SCATTER_RING>(a, s, e0, warp, lane, s.node + buf * NB, s.rs + buf * NB,
                                                s.nup + buf * NB, s.ranks + buf * NB);
            __syncthreads();
            if (t == 0) {
                __threadfence();
                st_release_u32(a.tile_done + cur, a.epoch);
            }
            if (next >= 0) buf = nb;
        } else {
            // ---------------- conversion item ----------------
            const int4 c = __ldg(a.conv + (-cur - 1));
            if (next >= 0) {  // stage the next tile meanwhile (buffers the conversion does not use)
                prefetch_conn(a, next * kTileE, s.node + buf * NB, s.ranks + buf * NB, t);
                cp_commit();
            }
            // every tile that reduces into these rows has finished: tiles [c.z, c.w]
            {
                const int per = (c.w - c.z + 1 + kThreads / 32 - 1) / (kThreads / 32);
                const int lo = c.z + warp * per, hi = min(c.w + 1, lo + per);
                if (hi > lo && !warp_wait_flags(a.tile_done, lo, hi, a.epoch, lane, a.sched_err) && lane == 0)
                    s_abort = 1;
            }
            if (next >= 0) cp_wait_all();
            __syncthreads();
            if (s_abort) break;
            if (next >= 0) {
                prefetch_nodes_state(a, next * kTileE, s.node + buf * NB, s.x, s.u, s.rs + buf * NB, s.nup + buf * NB,
                                     s.st, t, s.pe);
                cp_commit();
            }
            convert_rows<1>(a, c.x, c.y, stage, conv_info, t);  // one block in flight: no spills here
            __syncthreads();
            if (t == 0) {
                __threadfence();
                st_release_u32(a.conv_done + (-cur - 1), a.epoch);
            }
        }
        if (t == 0) s_item[slot] = item_at(requested);
        __syncthreads();
        cur = next;
        next = s_item[slot];
        slot ^= 1;
    }
    cp_wait_all();
}

}  // namespace ceos
