/*
 * ceos_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the CEOS (m-dalbosco/CEOS-EEMS) Newton-iteration element
 * loop, used as the parity checker for the sm_100a kernels.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product
 * library never links or calls it.
 *
 * Parity pinning: the restated element loop, upper-CSR assembly, rearrangement BCs
 * and Newton driver are checked against the reference's only golden Hexa8 case
 * (Checker/Cases/NonLinear_FEA_3D_Hexa8_StVenant: MARC displacement curves, Newton
 * counts and per-iteration norms), committed as tests/golden/hexa8_svk.json.
 * The CNH, J2 and viscoelastic restatements have no reference golden vectors; they are
 * pinned by closed-form known-answer tests and finite-difference tangent checks.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Material model ids.  1..16 are the reference registry ids
 * (ConstitutiveModelsLibrary/ModConstitutiveModelLibrary.f90:39-56); 101+ are
 * project-defined models with no reference implementation. */
enum {
    OR_J2_SMALL = 2,     /* ModJ2Plasticity.f90 (small strain, reference)           */
    OR_NH_Q1P0 = 4,      /* ModNeoHookeanQ1P0.f90 with the Mean Dilatation element  */
    OR_SVK = 5,          /* ModStVenantKirchhoff.f90                                 */
    OR_CNH = 7,          /* ModCompressibleNeoHookean.f90                            */
    OR_VISCO_VAR = 12,   /* ModViscoelasticMatrix.f90 (variational, one branch)      */
    OR_VISCO_PRONY = 101,/* finite-strain generalized Maxwell (Holzapfel 2000 6.10) */
    OR_J2_FINITE = 102   /* multiplicative J2 in b_e (Simo 1988; Simo-Hughes 9.1)  */
};

/* Number of parameters each model reads (per material or per element). */
int or_model_nparams(int model);
/* Number of FP64 state variables each model keeps per Gauss point. */
int or_model_nstate(int model);
/* Initial (virgin) state of one Gauss point. */
void or_model_init_state(int model, const double* params, double* st);

/* Material point update: F (row-major 3x3) -> Cauchy stress (Voigt 11,22,33,12,23,13),
 * spatial tangent D (6x6 row-major, full) and new state.  Returns 0 or a status code
 * (2 = local Newton not converged).  dt = time - time_old. */
int or_material_point(int model, const double* params, const double* F, double dt,
                      const double* st_old, double* st_new, double* sigma, double* D);

/* CSR pattern, restating ModFEMAnalysis.f90:209-273 with SparseMatrixSetArray and
 * ConvertToCoordinateFormatUpperTriangular (1-based, upper triangle, sorted columns). */
long long or_pattern_nnz(int n_nodes, int n_elem, const int* conn);
void or_pattern_fill(int n_nodes, int n_elem, const int* conn, int* rowmap, int* col, int* row);

/* Slot map: for each element and local pair (i,j) with GM(j) >= GM(i), the 0-based
 * CSR position found by the reference's linear search
 * (SubAssembleGlobalMatrixUpperTriangular.f90:43-65).  Entries with GM(j) < GM(i) are -1.
 * out: n_elem*24*24 int64. */
void or_slot_map(int n_nodes, int n_elem, const int* conn, const int* rowmap, const int* col,
                 long long* out);

/* ---------------------------------------------------------------------------------------- */
/* Model object: mesh + materials + per-GP state.                                          */
typedef struct or_model or_model;

/* X: [3*n_nodes] reference coordinates; conn: [8*n_elem] 1-based; mat_id [n_elem] 0-based
 * index into the material table.  models[n_mat]; params: if per_element==0,
 * [n_mat][n_params_max] else [n_elem][n_params_max] (model of each element still from
 * models[mat_id]). */
or_model* or_create(int n_nodes, int n_elem, const double* X, const int* conn,
                    const int* mat_id, int n_mat, const int* models, int per_element,
                    int n_params_max, const double* params);
void or_destroy(or_model* m);
long long or_nnz(or_model* m);
void or_get_pattern(or_model* m, int* rowmap, int* col);

/* One Newton evaluation: SolveConstitutiveModel + InternalForce (+ TangentStiffnessMatrix
 * when kval != NULL), reference semantics.  Returns 0 or the first error status;
 * n_failed receives the number of failed elements; failed_ids (size n_elem) gets their
 * 1-based ids when not NULL. */
int or_evaluate(or_model* m, double time, const double* U, double* fint, double* kval,
                int* n_failed, int* failed_ids);
/* Same, but only the first n_eval elements (CPU-baseline sampling).  threads>1 colours the
 * elements and runs them on OpenMP threads. */
int or_evaluate_sample(or_model* m, double time, const double* U, double* fint, double* kval,
                       int n_eval, int threads);
void or_commit(or_model* m);            /* SwitchConvergedState for every GP */
/* HomogenizeStress (ModMultiscaleAnalysis.f90:140-329) of the last evaluation: P row-major 3x3. */
void or_homogenize(or_model* m, const double* U, double* P_out);
/* Gauss-point results of the last evaluation: sigma [n_elem*8*6], state [n_elem*8*nstate]. */
void or_get_gp_stress(or_model* m, double* sigma);
int  or_get_state(or_model* m, double* st, int which /*0 old, 1 new*/);
int  or_set_state(or_model* m, const double* st, int which);
void or_set_time_old(or_model* m, double t);

/* Quasi-static analysis: QuasiStaticAnalysisFEM (ModFEMAnalysis.f90:1136-1374) +
 * NewtonRaphsonFull_Solve (ModNewtonRaphsonFull.f90:44-168) +
 * ApplyBoundaryConditionsNEW (ModBoundaryConditions.f90:246-340), one load case.
 *  step_t0/step_dt: [n_steps]; *_init/_final: [n_items*n_steps] (item-major);
 *  dofs are 1-based; norm_mode 0 = relative (current source), 1 = absolute (golden logs);
 *  norm_type 2 = max-abs (reference default), 1 = L2.
 *  iters[n_steps] = Newton iterations of the last (alpha = 1) substep of each step;
 *  cutbacks[n_steps]; probe_out[n_probe*n_steps] = U at probe dofs after each step;
 *  norm_log[max_log] = every printed NORM, n_log = count.  Returns 0 or -1 on failure. */
int or_analysis(or_model* m, int n_steps, const double* step_t0, const double* step_dt,
                int n_fixed, const int* fixed_dofs,
                int n_presc, const int* presc_dofs, const double* presc_init, const double* presc_final,
                int n_force, const int* force_dofs, const double* force_init, const double* force_final,
                double tol, int itmax, int norm_mode, int norm_type, int max_cutbacks,
                int* iters, int* cutbacks, int n_probe, const int* probe_dofs, double* probe_out,
                int max_log, double* norm_log, int* n_log, double* U_final);

#ifdef __cplusplus
}
#endif
