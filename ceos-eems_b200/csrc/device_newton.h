// device_newton.h -- device-resident Newton iteration used by ceos_analysis (device_newton.cu).
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "ceos_handle.h"

namespace ceos {

struct DeviceNewton {
    Handle* h = nullptr;
    int n = 0;
    long long n_zero = 0, n_one = 0;
    bool any_presc = false;
    void* pcg = nullptr;
    double *dX = nullptr, *dfint = nullptr, *dR = nullptr, *dUd = nullptr, *dDX = nullptr, *db = nullptr;
    double *dFext = nullptr, *dUbar = nullptr, *dtmp = nullptr, *dnorm = nullptr;
    uint8_t* dkind = nullptr;       // per dof bits: 1 prescribed, 2 fixed (0: free)
    int* dcol1 = nullptr;           // 1-based CSR columns
    long long *dzero = nullptr, *done = nullptr;  // K positions set to 0 / to 1 by the boundary conditions

    // kind: per dof bits 1 prescribed, 2 fixed; zero_pos: K positions in a constrained row or column
    // off its diagonal; one_pos: diagonals of constrained dofs (the two lists are disjoint)
    int setup(Handle* h, const std::vector<uint8_t>& kind, const std::vector<int>& col1,
              const std::vector<long long>& zero_pos, const std::vector<long long>& one_pos);
    // F_ext and Ubar of the current substep, and the starting iterate X
    int set_targets(const double* Fext, const double* Ubar, const double* X);
    // evaluation at X, boundary conditions and the residual norm; *status > 0 on an element failure
    int residual(double time, int it, int norm_type, double* norm, int* status);
    // K DX = -R and X += DX
    int solve_and_update(double tol, int max_iter, int* lin_iters);
    int get_X(double* X);
    ~DeviceNewton();
};

}  // namespace ceos
