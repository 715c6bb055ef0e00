// device_newton.cu -- the Newton iteration of ceos_analysis with the system kept on the device.
//
// The reference's host (FEM/Modules/ModFEMSystemOfEquations.f90:40-93 with
// Tools/MathTools/NonlinearSolver/ModNewtonRaphsonFull.f90:44-168) applies the boundary conditions
// to the assembled system (ApplyBoundaryConditionsNEW, FEM/BoundaryConditions/
// ModBoundaryConditions.f90:246-340) and hands it to PARDISO (ModPardisoSolver.f90:343-380).  Here
// every step of that iteration runs on the device, so K (hundreds of MB on the benchmark meshes)
// never crosses PCIe:
//   residual   R = -(f_int - F_ext)
//   it = 0     Ud = Ubar - X on the prescribed dofs, R -= K Ud (mkl_dcsrsymv 'U' on the upper CSR,
//              :289-333)
//   masks      K entries in a constrained row or column = 0, their diagonal = 1 (the positions of
//              AllocatePrescDispSparseMapping / AllocateFixedSupportSparseMapping, :344-536),
//              R = Ud on prescribed dofs, 0 on fixed dofs; R = -R
//   norm       max |R_i| or ||R||_2 (ModNewtonRaphsonFull.f90:109-125), 8 bytes to the host
//   solve      K DX = -R: block-Jacobi PCG on the free dofs (the constrained rows are identity
//              with zero coupling after the masks, so DX_c = -R_c there), then X += DX.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/ceos_gpu.h"
#include "ceos_handle.h"
#include "device_newton.h"

namespace {

__device__ __forceinline__ long long dn_row_start(const long long* rs, const int* nup, int row, int* len) {
    const int a = row / 3, k = row - 3 * a, m = nup[a];
    *len = (3 - k) + 3 * m;
    return rs[a] + (k == 0 ? 0LL : (k == 1 ? 3LL + 3LL * m : 5LL + 6LL * m));
}

// kind bits per dof: 1 prescribed, 2 fixed (either makes the dof constrained)
constexpr uint8_t kPresc = 1, kFixed = 2;

// R = Fext - fint; at it = 0 also Ud = Ubar - X on the prescribed dofs (0 elsewhere)
__global__ void dn_residual_kernel(int n, const double* fint, const double* Fext, const double* X, const double* Ubar,
                                   const uint8_t* kind, int first_it, double* R, double* Ud) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    R[i] = -(fint[i] - Fext[i]);
    if (first_it) Ud[i] = (kind[i] & kPresc) ? Ubar[i] - X[i] : 0.0;
}

// y = K x for the symmetric K stored as its upper CSR; warp per row, transposed half by atomics
__global__ void dn_symv_kernel(int n, const long long* rs, const int* nup, const int* col1, const double* K,
                               const double* x, double* y) {
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= n) return;
    int len;
    const long long start = dn_row_start(rs, nup, row, &len);
    const double xr = x[row];
    double acc = 0.0;
    for (int t = lane; t < len; t += 32) {
        const int c = col1[start + t] - 1;
        const double v = K[start + t];
        acc += v * x[c];
        if (c != row && xr != 0.0) atomicAdd(y + c, v * xr);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) atomicAdd(y + row, acc);
}

__global__ void dn_sub_kernel(int n, const double* a, double* R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) R[i] -= a[i];
}

// K[pos] = 0 in constrained rows/columns off their diagonal, 1 on their diagonal (disjoint lists)
__global__ void dn_mask_kernel(long long n_zero, const long long* zero_pos, long long n_one, const long long* one_pos,
                               double* K) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n_zero) K[zero_pos[i]] = 0.0;
    if (i < n_one) K[one_pos[i]] = 1.0;
}

// constrained entries of R, sign flip, b = -R for the solve, and the residual norm
__global__ void dn_finish_kernel(int n, const uint8_t* kind, const double* Ud, int first_it, int norm_type, double* R,
                                 double* b, unsigned long long* norm_bits, double* norm_sum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        double r = R[i];
        if (kind[i] & kPresc) r = first_it ? Ud[i] : 0.0;  // Ud is zero after the first iteration
        if (kind[i] & kFixed) r = 0.0;
        r = -r;
        R[i] = r;
        b[i] = -r;
        v = r;
    }
    if (norm_type == 2) {
        double m = fabs(v);
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) atomicMax(norm_bits, (unsigned long long)__double_as_longlong(m));
    } else {
        double s = v * v;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(norm_sum, s);
    }
}

// DX_c = b_c on constrained dofs (identity rows), X += DX
__global__ void dn_update_kernel(int n, const uint8_t* kind, const double* b, double* DX, double* X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kind[i]) DX[i] = b[i];
    X[i] += DX[i];
}

}  // namespace

namespace ceos {

#define CKD(call)                                 \
    do {                                          \
        if ((call) != cudaSuccess) {              \
            h->msg = "device Newton: " #call;     \
            return CEOS_E_CUDA;                   \
        }                                         \
    } while (0)

DeviceNewton::~DeviceNewton() {
    if (pcg) ceos_pcg_destroy(pcg);
    void* ptrs[] = {dX, dfint, dR, dUd, dDX, db, dFext, dUbar, dtmp, dkind, dcol1, dzero, done, dnorm};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

int DeviceNewton::setup(Handle* hh, const std::vector<uint8_t>& kind, const std::vector<int>& col1,
                        const std::vector<long long>& zero_pos, const std::vector<long long>& one_pos) {
    h = hh;
    n = 3 * h->n_nodes;
    n_zero = (long long)zero_pos.size();
    n_one = (long long)one_pos.size();
    any_presc = false;
    for (uint8_t k : kind) any_presc |= (k & kPresc) != 0;
    CKD(cudaSetDevice(h->device));
    const size_t nb = sizeof(double) * n;
    double** vecs[] = {&dX, &dfint, &dR, &dUd, &dDX, &db, &dFext, &dUbar, &dtmp};
    for (double** v : vecs) CKD(cudaMalloc(v, nb));
    CKD(cudaMalloc(&dkind, n));
    CKD(cudaMemcpy(dkind, kind.data(), n, cudaMemcpyHostToDevice));
    CKD(cudaMalloc(&dcol1, sizeof(int) * col1.size()));
    CKD(cudaMemcpy(dcol1, col1.data(), sizeof(int) * col1.size(), cudaMemcpyHostToDevice));
    CKD(cudaMalloc(&dzero, sizeof(long long) * (n_zero + 1)));
    CKD(cudaMalloc(&done, sizeof(long long) * (n_one + 1)));
    if (n_zero) CKD(cudaMemcpy(dzero, zero_pos.data(), sizeof(long long) * n_zero, cudaMemcpyHostToDevice));
    if (n_one) CKD(cudaMemcpy(done, one_pos.data(), sizeof(long long) * n_one, cudaMemcpyHostToDevice));
    CKD(cudaMalloc(&dnorm, 16));
    const int rc = ceos_pcg_create(h, &pcg);
    if (rc) return rc;
    return 0;
}

int DeviceNewton::set_targets(const double* Fext, const double* Ubar, const double* X) {
    CKD(cudaMemcpyAsync(dFext, Fext, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CKD(cudaMemcpyAsync(dUbar, Ubar, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CKD(cudaMemcpyAsync(dX, X, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    return 0;
}

int DeviceNewton::residual(double time, int it, int norm_type, double* norm, int* status) {
    cudaStream_t s = h->stream;
    int rc = evaluate_device(h, time, dX, dfint, h->d_kval, s);
    if (rc) return rc;
    int nfail = 0;
    const int st = ceos_status(h, &nfail);  // synchronizes
    if (st < 0) return st;
    *status = st;
    if (st) return 0;
    const int first = it == 0 ? 1 : 0;
    const unsigned g = (unsigned)((n + 255) / 256);
    dn_residual_kernel<<<g, 256, 0, s>>>(n, dfint, dFext, dX, dUbar, dkind, first, dR, dUd);
    if (first && any_presc) {  // R -= K Ud with the unmodified K
        CKD(cudaMemsetAsync(dtmp, 0, sizeof(double) * n, s));
        dn_symv_kernel<<<(unsigned)(((long long)n * 32 + 255) / 256), 256, 0, s>>>(n, h->d_rs, h->d_nup, dcol1,
                                                                                   h->d_kval, dUd, dtmp);
        dn_sub_kernel<<<g, 256, 0, s>>>(n, dtmp, dR);
    }
    const long long nm = n_zero > n_one ? n_zero : n_one;
    if (nm) dn_mask_kernel<<<(unsigned)((nm + 255) / 256), 256, 0, s>>>(n_zero, dzero, n_one, done, h->d_kval);
    CKD(cudaMemsetAsync(dnorm, 0, 16, s));
    dn_finish_kernel<<<g, 256, 0, s>>>(n, dkind, dUd, first, norm_type, dR, db,
                                       reinterpret_cast<unsigned long long*>(dnorm), dnorm + 1);
    CKD(cudaGetLastError());
    double hn[2];
    CKD(cudaMemcpyAsync(hn, dnorm, 16, cudaMemcpyDeviceToHost, s));
    CKD(cudaStreamSynchronize(s));
    *norm = norm_type == 2 ? hn[0] : std::sqrt(hn[1]);
    return 0;
}

int DeviceNewton::solve_and_update(double tol, int max_iter, int* lin_iters) {
    double rel = 0.0;
    const int rc = ceos_pcg_solve(pcg, h->d_kval, dkind, db, dDX, tol, max_iter, lin_iters, &rel);
    if (rc) return rc;
    dn_update_kernel<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(n, dkind, db, dDX, dX);
    CKD(cudaGetLastError());
    return 0;
}

int DeviceNewton::get_X(double* X) {
    CKD(cudaMemcpyAsync(X, dX, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CKD(cudaStreamSynchronize(h->stream));
    return 0;
}

}  // namespace ceos
