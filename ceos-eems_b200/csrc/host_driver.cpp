// host_driver.cpp -- the host side above the C ABI: quasi-static increments, full Newton and
// the rearrangement boundary conditions of the reference's Fortran host, restated in C++ so
// that Newton histories can be driven through ceos_evaluate.  PARDISO (phase 13 per iteration,
// Tools/MathTools/LinearSolver/ModPardisoSolver.f90:343-380) is replaced by a skyline LDL^T on a
// reverse Cuthill-McKee node ordering.
#include <algorithm>
#include <cmath>
#include <deque>
#include <memory>
#include <vector>

#include "../../include/ceos_gpu.h"
#include "ceos_handle.h"
#include "device_newton.h"

namespace {

using ceos::Handle;

// Reverse Cuthill-McKee ordering of the node graph given by the upper-neighbour lists.
std::vector<int> rcm_nodes(const Handle* h) {
    const int N = h->n_nodes;
    std::vector<std::vector<int>> adj(N);
    for (int n = 0; n < N; ++n)
        for (long long q = h->up_ptr[n]; q < h->up_ptr[n + 1]; ++q) {
            adj[n].push_back(h->up_list[q]);
            adj[h->up_list[q]].push_back(n);
        }
    std::vector<int> order;
    order.reserve(N);
    std::vector<char> seen(N, 0);
    for (int comp_start = 0; (int)order.size() < N;) {
        // lowest-degree unvisited node starts the next component
        int s = -1;
        for (int n = 0; n < N; ++n)
            if (!seen[n] && (s < 0 || adj[n].size() < adj[s].size())) s = n;
        std::deque<int> q{s};
        seen[s] = 1;
        while (!q.empty()) {
            const int v = q.front();
            q.pop_front();
            order.push_back(v);
            std::vector<int> nb;
            for (int w : adj[v])
                if (!seen[w]) { seen[w] = 1; nb.push_back(w); }
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
            for (int w : nb) q.push_back(w);
        }
        (void)comp_start;
    }
    std::reverse(order.begin(), order.end());
    std::vector<int> newid(N);
    for (int i = 0; i < N; ++i) newid[order[i]] = i;
    return newid;
}

// Variable-band (skyline) symmetric LDL^T in the permuted numbering.
struct SkylineLDLT {
    int n = 0;
    std::vector<int> perm;           // old dof -> new dof
    std::vector<int> first;          // first row of column j
    std::vector<long long> start;    // column j occupies [start[j], start[j+1]) rows first..j
    std::vector<double> v;
    bool ok = false;

    void analyse(const Handle* h) {
        n = 3 * h->n_nodes;
        const std::vector<int> nid = rcm_nodes(h);
        perm.resize(n);
        for (int nd = 0; nd < h->n_nodes; ++nd)
            for (int d = 0; d < 3; ++d) perm[3 * nd + d] = 3 * nid[nd] + d;
        first.assign(n, 0);
        for (int j = 0; j < n; ++j) first[j] = j;
        for (int nd = 0; nd < h->n_nodes; ++nd)
            for (long long q = h->up_ptr[nd]; q < h->up_ptr[nd + 1]; ++q) {
                const int a = nid[nd], b = nid[h->up_list[q]];
                const int lo = std::min(a, b), hi = std::max(a, b);
                for (int d = 0; d < 3; ++d) first[3 * hi + d] = std::min(first[3 * hi + d], 3 * lo);
            }
        for (int nd = 0; nd < h->n_nodes; ++nd)
            for (int d = 0; d < 3; ++d) first[3 * nid[nd] + d] = std::min(first[3 * nid[nd] + d], 3 * nid[nd]);
        start.assign(n + 1, 0);
        for (int j = 0; j < n; ++j) start[j + 1] = start[j] + (j - first[j] + 1);
        v.assign(start[n], 0.0);
    }
    double& a(int i, int j) { return v[start[j] + (i - first[j])]; }

    bool factor(const Handle* h, const int* rowmap, const int* col, const double* val) {
        std::fill(v.begin(), v.end(), 0.0);
        for (int r = 0; r < n; ++r)
            for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
                const int i = perm[r], j = perm[col[k] - 1];
                a(std::min(i, j), std::max(i, j)) += val[k];
            }
        (void)h;
        for (int j = 0; j < n; ++j) {
            const int fj = first[j];
            double* cj = &v[start[j]];  // cj[i - fj]
            for (int i = fj; i < j; ++i) {
                const int fi = first[i];
                const int k0 = std::max(fi, fj);
                const double* ci = &v[start[i]];
                double s = 0.0;
                for (int k = k0; k < i; ++k) s += ci[k - fi] * cj[k - fj];
                cj[i - fj] -= s;
            }
            double d = cj[j - fj];
            for (int i = fj; i < j; ++i) {
                const double g = cj[i - fj];
                const double l = g / v[start[i] + (i - first[i])];
                d -= l * g;
                cj[i - fj] = l;
            }
            if (!(std::fabs(d) > 0.0) || !std::isfinite(d)) return ok = false;
            cj[j - fj] = d;
        }
        return ok = true;
    }
    void solve(const double* b, double* x) {
        std::vector<double> y(n);
        for (int r = 0; r < n; ++r) y[perm[r]] = b[r];
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int i = first[j]; i < j; ++i) s += a(i, j) * y[i];
            y[j] -= s;
        }
        for (int j = 0; j < n; ++j) y[j] /= a(j, j);
        for (int j = n - 1; j >= 0; --j)
            for (int i = first[j]; i < j; ++i) y[i] -= a(i, j) * y[j];
        for (int r = 0; r < n; ++r) x[r] = y[perm[r]];
    }
};

// y = K x, K symmetric stored as its upper triangle (mkl_dcsrsymv 'U', ModBoundaryConditions.f90:300)
void symv_upper(int n, const int* rowmap, const int* col, const double* val, const double* x, double* y) {
    std::fill(y, y + n, 0.0);
    for (int r = 0; r < n; ++r)
        for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
            const int c = col[k] - 1;
            y[r] += val[k] * x[c];
            if (c != r) y[c] += val[k] * x[r];
        }
}

}  // namespace

extern "C" int ceos_analysis_set_callback(void* handle, ceos_step_callback cb, void* user) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    h->step_cb = cb;
    h->step_user = cb ? user : nullptr;
    return 0;
}

extern "C" int ceos_analysis_set_initial(void* handle, const double* U0) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return CEOS_E_ARG;
    if (U0)
        h->U_start.assign(U0, U0 + 3 * (size_t)h->n_nodes);
    else
        h->U_start.clear();
    return 0;
}

extern "C" int ceos_analysis_set_device_solver(void* handle, int on, double lin_tol, int lin_max_iter) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || (on && (!(lin_tol > 0.0) || lin_max_iter < 1))) return CEOS_E_ARG;
    h->device_newton = on != 0;
    h->lin_tol = lin_tol;
    h->lin_max_iter = lin_max_iter;
    return 0;
}

extern "C" int ceos_analysis(void* handle, int n_steps, const double* step_t0, const double* step_dt, int n_fixed,
                             const int* fixed_dofs, int n_presc, const int* presc_dofs, const double* presc_init,
                             const double* presc_final, int n_force, const int* force_dofs, const double* force_init,
                             const double* force_final, double tol, int itmax, int norm_mode, int norm_type,
                             int max_cutbacks, int* iters, int* cutbacks, int n_probe, const int* probe_dofs,
                             double* probe_out, int max_log, double* norm_log, int* n_log, double* U_final) {
    Handle* h = static_cast<Handle*>(handle);
    if (!h || n_steps < 1) return CEOS_E_ARG;
    const int n = 3 * h->n_nodes;
    const long long nnz = h->nnz;
    std::vector<int> rowmap(n + 1), col(nnz);
    int rc = ceos_pattern(handle, nullptr, nullptr, rowmap.data(), col.data(), nullptr);
    if (rc) return rc;
    // masks of AllocatePrescDispSparseMapping / AllocateFixedSupportSparseMapping
    // (ModBoundaryConditions.f90:344-536): entries in a constrained row or column, and diagonals
    std::vector<char> is_presc(n, 0), is_fixed(n, 0);
    for (int i = 0; i < n_presc; ++i) is_presc[presc_dofs[i] - 1] = 1;
    for (int i = 0; i < n_fixed; ++i) is_fixed[fixed_dofs[i] - 1] = 1;
    std::vector<long long> zp, op, zf, of;
    for (int r = 0; r < n; ++r)
        for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
            const int c = col[k] - 1;
            if (is_presc[r] || is_presc[c]) zp.push_back(k);
            if (is_presc[r] && c == r) op.push_back(k);
            if (is_fixed[r] || is_fixed[c]) zf.push_back(k);
            if (is_fixed[r] && c == r) of.push_back(k);
        }
    // device-resident Newton (ceos_analysis_set_device_solver): the same boundary conditions as
    // kernels, K stays on the device and a PCG replaces the host factorization
    std::unique_ptr<ceos::DeviceNewton> dn;
    SkylineLDLT lin;
    if (h->device_newton) {
        std::vector<uint8_t> kind(n, 0);
        for (int r = 0; r < n; ++r) kind[r] = (uint8_t)((is_presc[r] ? 1 : 0) | (is_fixed[r] ? 2 : 0));
        std::vector<long long> zero_pos, one_pos;
        for (int r = 0; r < n; ++r)
            for (int k = rowmap[r] - 1; k < rowmap[r + 1] - 1; ++k) {
                const int c = col[k] - 1;
                if (!kind[r] && !kind[c]) continue;
                (c == r ? one_pos : zero_pos).push_back(k);
            }
        dn.reset(new ceos::DeviceNewton());
        rc = dn->setup(h, kind, col, zero_pos, one_pos);
        if (rc) return rc;
    } else {
        lin.analyse(h);
    }
    std::vector<double> U(n, 0.0), Uconv(n), Ubar(n), Ubar0(n), Fext(n), Fext0(n), dFext(n), dUp(n);
    if (!h->U_start.empty()) {  // restart: U of the last converged step
        if ((int)h->U_start.size() != n) return CEOS_E_ARG;
        U = h->U_start;
        h->U_start.clear();
    }
    std::vector<double> X(n), R(n), fint(n), kval(nnz), DX(n), Ud(n), Rmod(n), mR(n);
    const double GR = (1.0 + std::sqrt(5.0)) / 2.0;
    int nl = 0;
    for (int ST = 0; ST < n_steps; ++ST) {
        std::fill(Fext0.begin(), Fext0.end(), 0.0);
        std::fill(dFext.begin(), dFext.end(), 0.0);
        for (int i = 0; i < n_force; ++i) {
            const size_t q = (size_t)i * n_steps + ST;
            Fext0[force_dofs[i] - 1] += force_init[q];
            dFext[force_dofs[i] - 1] += force_final[q] - force_init[q];
        }
        std::fill(dUp.begin(), dUp.end(), 0.0);
        for (int i = 0; i < n_presc; ++i) {
            const size_t q = (size_t)i * n_steps + ST;
            U[presc_dofs[i] - 1] = presc_init[q];
            dUp[presc_dofs[i] - 1] = presc_final[q] - presc_init[q];
        }
        Ubar0 = U;
        Uconv = U;
        double alpha = 1.0, alpha_min = 0.0, alpha_aux;
        int CutBack = 0, SubStep = 0;
        while (true) {
            const double Time = step_t0[ST] + alpha * step_dt[ST];
            for (int i = 0; i < n; ++i) {
                Fext[i] = Fext0[i] + alpha * dFext[i];
                Ubar[i] = Ubar0[i] + alpha * dUp[i];
            }
            X = Uconv;
            int it = 0;
            double normR0 = 0.0;
            bool converged = false;
            if (dn) {
                rc = dn->set_targets(Fext.data(), Ubar.data(), X.data());
                if (rc) return rc;
            }
            while (dn) {
                double normR = 0.0;
                int st = 0;
                rc = dn->residual(Time, it, norm_type, &normR, &st);
                if (rc) return rc;
                if (st) break;  // element failure: cut back
                if (nl < max_log && norm_log) norm_log[nl] = normR;
                ++nl;
                if (it == 0) normR0 = normR;
                const double thr = norm_mode == 0 ? normR0 * tol : tol;
                if (it > 0 && normR < thr) {
                    converged = true;
                    rc = dn->get_X(X.data());
                    if (rc) return rc;
                    break;
                }
                if (it >= itmax) break;
                ++it;
                int lin_iters = 0;
                rc = dn->solve_and_update(h->lin_tol, h->lin_max_iter, &lin_iters);
                if (rc == CEOS_E_SOLVER) break;  // no converged correction: cut back as on a singular system
                if (rc) return rc;
            }
            while (!dn) {
                int nfail = 0;
                const int st = ceos_evaluate(handle, Time, X.data(), fint.data(), kval.data(), &nfail);
                if (st < 0) return st;
                if (st) break;  // element failure: cut back
                for (int i = 0; i < n; ++i) R[i] = -(fint[i] - Fext[i]);
                std::fill(Ud.begin(), Ud.end(), 0.0);
                if (n_presc) {
                    if (it == 0) {
                        for (int i = 0; i < n_presc; ++i) {
                            const int d = presc_dofs[i] - 1;
                            Ud[d] = Ubar[d] - X[d];
                        }
                        symv_upper(n, rowmap.data(), col.data(), kval.data(), Ud.data(), Rmod.data());
                        for (int i = 0; i < n; ++i) R[i] -= Rmod[i];
                    }
                    for (long long k : zp) kval[k] = 0.0;
                    for (long long k : op) kval[k] = 1.0;
                    for (int i = 0; i < n_presc; ++i) R[presc_dofs[i] - 1] = Ud[presc_dofs[i] - 1];
                }
                if (n_fixed) {
                    for (long long k : zf) kval[k] = 0.0;
                    for (long long k : of) kval[k] = 1.0;
                    for (int i = 0; i < n_fixed; ++i) R[fixed_dofs[i] - 1] = 0.0;
                }
                for (int i = 0; i < n; ++i) R[i] = -R[i];
                double normR = 0.0;
                if (norm_type == 2) {
                    for (int i = 0; i < n; ++i) normR = std::max(normR, std::fabs(R[i]));
                } else {
                    for (int i = 0; i < n; ++i) normR += R[i] * R[i];
                    normR = std::sqrt(normR);
                }
                if (nl < max_log && norm_log) norm_log[nl] = normR;
                ++nl;
                if (it == 0) normR0 = normR;
                const double thr = norm_mode == 0 ? normR0 * tol : tol;
                if (it > 0 && normR < thr) { converged = true; break; }
                if (it >= itmax) break;
                ++it;
                if (!lin.factor(h, rowmap.data(), col.data(), kval.data())) break;
                for (int i = 0; i < n; ++i) mR[i] = -R[i];
                lin.solve(mR.data(), DX.data());
                for (int i = 0; i < n; ++i) X[i] += DX[i];
            }
            if (!converged) {
                alpha = alpha_min + (1.0 - 1.0 / GR) * (alpha - alpha_min);
                ++CutBack;
                SubStep = 1;
                if (CutBack > max_cutbacks) {
                    if (n_log) *n_log = nl;
                    return -10;
                }
                continue;
            }
            U = X;
            ++SubStep;
            if (alpha == 1.0) {
                if (iters) iters[ST] = it;
                if (cutbacks) cutbacks[ST] = CutBack;
                if (h->step_cb && h->step_cb(h->step_user, Time, 1, ST + 1, CutBack, SubStep, 1, it, n, U.data())) {
                    if (n_log) *n_log = nl;
                    return CEOS_E_ABORTED;
                }
                break;
            }
            alpha_aux = alpha_min;
            alpha_min = alpha;
            alpha = std::min(alpha + GR * (alpha - alpha_aux), 1.0);
            Uconv = U;
            if (h->step_cb && h->step_cb(h->step_user, Time, 1, ST + 1, CutBack, SubStep, 0, it, n, U.data())) {
                if (n_log) *n_log = nl;
                return CEOS_E_ABORTED;
            }
        }
        // SwitchConvergedState; the evaluation time of the last converged iteration is committed
        rc = ceos_commit_state(handle);
        if (rc) return rc;
        ceos_set_committed_time(handle, step_t0[ST] + step_dt[ST]);
        for (int p = 0; p < n_probe; ++p) probe_out[(size_t)p * n_steps + ST] = U[probe_dofs[p] - 1];
    }
    if (n_log) *n_log = nl;
    if (U_final) std::copy(U.begin(), U.end(), U_final);
    return 0;
}
