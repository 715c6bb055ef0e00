/*
 * ceos_gpu.h -- C ABI of the B200 (sm_100a) element loop for CEOS.
 *
 * Replaces, as a drop-in, the three serial passes that the CEOS Newton "system of
 * equations" plugin runs per iteration (reference paths relative to SourceCode/):
 *   SolveConstitutiveModel  FEM/Subroutines/SubSolveConstitutiveModel.f90:13
 *   InternalForce           FEM/Subroutines/SubInternalForce.f90:13
 *   TangentStiffnessMatrix  FEM/Subroutines/SubTangentStiffnessMatrix.f90:13 (FEM branch :294-311)
 *     + AssembleGlobalMatrixUpperTriangular  FEM/Subroutines/SubAssembleGlobalMatrixUpperTriangular.f90:13
 * as called by EvaluateR / EvaluateKt (FEM/Modules/ModFEMSystemOfEquations.f90:40-93), and the
 * CSR allocation AllocateKgSparseUpperTriangular (FEM/ModFEMAnalysis.f90:209-273).
 *
 * Conventions follow the reference's ClassGlobalSparseMatrix (Tools/MathTools/
 * SparseMatrixRoutines/ModGlobalSparseMatrix.f90:18-25): DOF order 3*(node-1)+d, 1-based
 * CSR of the upper triangle with sorted columns, real(8) values, as PARDISO consumes them.
 * All ints are 32-bit except nnz and slot positions (64-bit).  All pointers are host
 * pointers unless the name says _device.  One host thread per handle.
 *
 * Return codes mirror ClassStatus (Tools/ModStatus.f90:3-49): 0 success;
 *   1 element geometry (det J <= 1e-13, ModElement.f90:555,1254,1396),
 *   2 local constitutive Newton not converged (ModViscoelasticMatrix.f90:565),
 *   3 non-finite stress;
 * negative values are usage, CUDA or allocation errors (CEOS_E_*).
 */
#ifndef CEOS_GPU_H
#define CEOS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Material model ids: reference registry ids (ConstitutiveModelsLibrary/
 * ModConstitutiveModelLibrary.f90:39-56) and project-defined models (>= 101). */
enum ceos_model_id {
    CEOS_J2_SMALL = 2,       /* ModJ2Plasticity.f90, params [E, nu, YieldStress, HardeningModulus]      */
    CEOS_NH_Q1P0 = 4,        /* ModNeoHookeanQ1P0.f90 on the Mean Dilatation Hexa8 (Jbar = V/V0 per      */
                             /* element, ModElement.f90:429-469), params [C10, BulkModulus]                */
    CEOS_SVK = 5,            /* ModStVenantKirchhoff.f90, params [YoungModulus, Poisson]                  */
    CEOS_CNH = 7,            /* ModCompressibleNeoHookean.f90, params [Mu, Lambda]                        */
    CEOS_VISCO_VAR = 12,     /* ModViscoelasticMatrix.f90, params [K_inf, Mu_inf, Lambda_inf, K_e, Mu_e, Ni_v] */
    CEOS_VISCO_PRONY = 101,  /* finite-strain generalized Maxwell, params [mu, K, nb, beta1, tau1, .. beta4, tau4] */
    CEOS_J2_FINITE = 102     /* multiplicative J2 (Simo 1988), params [E, nu, sigma_y0, H]                 */
};

enum ceos_precision {
    CEOS_FP64 = 0,   /* every operation in FP64 (the reference's real(8))                             */
    CEOS_MIXED = 1   /* FP32 element arithmetic and state; FP64 det F, ln J, return mapping, K, f_int */
};

enum ceos_error {
    CEOS_E_ARG = -1, CEOS_E_CUDA = -2, CEOS_E_ALLOC = -3, CEOS_E_MESH = -4, CEOS_E_MODEL = -5,
    CEOS_E_SOLVER = -6, /* iterative solver did not reach its tolerance */
    CEOS_E_ABORTED = -7 /* a step callback asked the analysis driver to stop */
};

/* Mesh as the reference holds it: CoordX interleaved [3*n_nodes] (ModNodes.f90:55),
 * connectivity [8*n_elem] 1-based in the Hexa8 node order (ModElementHexa8.f90:185-192),
 * mat_id [n_elem] 0-based into the material table (NULL: all 0). */
typedef struct ceos_mesh {
    int n_nodes, n_elem;
    const double* X;
    const int* conn;
    const int* mat_id;
} ceos_mesh;

/* One material (the reference's MaterialList entry, SubMaterialConstructor.f90:13-60).
 * per_element = 0: params[n_params] shared by every Gauss point of this material, as the
 * reference shares its Properties pointer (:58-60); per_element = 1: params[n_params*n_elem]
 * element-major (a build feature the reference does not have).  All materials of one
 * handle must use the same model id. */
typedef struct ceos_material {
    int model;
    int per_element;
    int n_params;
    const double* params;
} ceos_material;

/* Build the handle: uploads the mesh, builds the upper CSR pattern
 * (AllocateKgSparseUpperTriangular, ModFEMAnalysis.f90:209-273) and the element-to-CSR
 * slot map, allocates Gauss-point state (virgin state, ConstitutiveModelConstructor) and
 * one CUDA stream.  CEOS_MIXED also plans the K assembly (conversion items, the fused queue,
 * the bands) and caches the reference geometry of every Gauss point (J_X^-1 and det J_X,
 * computed in FP64, 320 bytes per element): the reference coordinates are fixed for the
 * handle's lifetime.  device = CUDA ordinal. */
int ceos_create(const ceos_mesh* mesh, const ceos_material* mats, int n_mat, int precision_mode,
                int device, void** handle);

/* Export the pattern: rowmap [n_dof+1], col [nnz], row [nnz] (Kg%RowMap, Kg%Col, Kg%Row),
 * 1-based.  Any array pointer may be NULL. */
int ceos_pattern(void* handle, int* n_dof, long long* nnz, int* rowmap, int* col, int* row);

/* Export the element-to-CSR slot map expanded to the reference's form: for element e and
 * local pair (i,j) with GM(j) >= GM(i), out[(e*24+i)*24+j] = 0-based position in Kg%Val that
 * AssembleGlobalMatrixUpperTriangular's linear search finds
 * (SubAssembleGlobalMatrixUpperTriangular.f90:43-65); -1 for GM(j) < GM(i). */
int ceos_slot_map(void* handle, long long* out);

/* One Newton evaluation (EvaluateR + the K part of EvaluateKt before BCs):
 * per Gauss point F, stress, state and tangent; f_int = sum_e B^T sigma; when kval != NULL,
 * Kg%Val = sum_e assembled (B^T D B + G^T S G).  Host buffers: U [n_dof], fint [n_dof],
 * kval [nnz] or NULL.  time is the reference's analysis time (dt = time - committed time).
 * n_failed (may be NULL) receives the number of failed elements.  Synchronous. */
int ceos_evaluate(void* handle, double time, const double* U, double* fint, double* kval, int* n_failed);

/* Same with device-resident buffers, enqueued on `stream` (NULL: the handle's stream);
 * asynchronous: the status is read by ceos_status() after the caller synchronizes. */
int ceos_evaluate_device(void* handle, double time, const double* U_device, double* fint_device,
                         double* kval_device, void* stream);
/* Status of the last evaluation: 0; when elements failed (n_failed of them; ceos_last_error names
 * them) the reference's ClassStatus code of the worst one (1 det J <= 1e-13, 2 a failed constitutive
 * update, 3 a non-finite stress); or CEOS_E_CUDA when a bounded wait of the mixed-precision K assembly
 * gave up (a dependency wait of the fused assembly or a block copy of the conversion pass; K is
 * incomplete and the next evaluation clears the FP32 blocks). */
int ceos_status(void* handle, int* n_failed);

/* SwitchConvergedState (ModFEMAnalysis.f90:1349-1353) for every Gauss point; the time of the
 * last evaluation becomes the committed time. */
int ceos_commit_state(void* handle);

/* Failed element ids (1-based, as ErrorElement.txt lists them, SubSolveConstitutiveModel.f90:69-83)
 * and a message for the last evaluation. */
int ceos_last_error(void* handle, int* elem_ids, int max_ids, char* msg, int msg_len);

/* Gauss-point state and stress access (host FP64 arrays [n_elem][8][nvars]); which = 0 for the
 * committed state, 1 for the state of the last evaluation.  ceos_gp_stress needs
 * ceos_set_options(handle, CEOS_OPT_STORE_STRESS) before the evaluation. */
int ceos_state_size(void* handle, int* nvars);
int ceos_get_state(void* handle, int which, double* out);
int ceos_set_state(void* handle, int which, const double* in);
int ceos_gp_stress(void* handle, double* out);
enum { CEOS_OPT_STORE_STRESS = 1, CEOS_OPT_TIME_KERNELS = 2 };
int ceos_set_options(void* handle, int options);
/* With CEOS_OPT_TIME_KERNELS set, CUDA events bracket the kernels of every evaluation; this
 * returns their device time (ms) for the last evaluation (synchronizes): ms[0] the element loop,
 * ms[1] the conversion of the FP32 node-pair blocks into the FP64 CSR rows (CEOS_MIXED two-pass
 * assembly; 0 when one launch does both or there is no conversion). */
int ceos_kernel_time(void* handle, float* ms);
/* CEOS_MIXED K assembly: CEOS_ASSEMBLY_TWO_PASS (default) runs the element loop, reducing FP32
 * node-pair blocks into a scratch array that holds all of them, then a conversion launch writes
 * the FP64 CSR rows; CEOS_ASSEMBLY_FUSED runs both in one launch from a host-planned queue, with
 * the blocks in a ring sized for L2; CEOS_ASSEMBLY_BANDED runs the two passes band by band, element
 * bands on two alternating streams and each band's conversion on a third, the blocks in a ring that
 * holds the rows of a few bands.  All give the same K up to the FP32 summation order. */
enum { CEOS_ASSEMBLY_TWO_PASS = 0, CEOS_ASSEMBLY_FUSED = 1, CEOS_ASSEMBLY_BANDED = 2 };
int ceos_set_assembly(void* handle, int mode);
/* Kernel launches of one device-resident evaluation (with or without a tangent) under the current
 * assembly. */
int ceos_launch_count(void* handle, int tangent, int* n_launches);
/* Failure-path test of the fused assembly: on != 0 makes conversion item `item` wait for a flag that
 * nothing sets, so its bounded wait (200 ms) runs out: the launch aborts, ceos_status reports
 * CEOS_E_CUDA and the next evaluation clears the blocks; on = 0 restores the item. */
int ceos_test_stall_conversion(void* handle, int item, int on);
int ceos_set_committed_time(void* handle, double t);

/* Release every device buffer and the stream. */
void ceos_destroy(void* handle);

/* Allocation-free assembly (no counterpart in the reference: CEOS assembles on the host).
 * For callers that cannot call cudaMalloc while they assemble, because the GPU memory belongs
 * to their own allocator or pool: one evaluation of the compressible Neo-Hookean element loop
 * (Gauss-point update, f_int, K into the upper CSR) in FP32 element arithmetic, taking only
 * caller-owned device buffers -- X [3*n_nodes] and U [3*n_nodes] (FP64), conn [8*n_elem]
 * (1-based), the 1-based upper CSR pattern rowmap [3*n_nodes+1] / col [nnz] exactly as
 * ceos_pattern exports it, outputs fint [3*n_nodes] and kval [nnz] (FP64) -- on the current
 * CUDA device and `stream` (NULL: default stream).  The FP32 node-pair block scratch is a static
 * 8 MiB device array inside the library (held by every GPU that loads it until exit), so a
 * call accepts at most 174,762 node pairs, i.e. n_nodes + (nnz - 6*n_nodes)/9 <= 174,762
 * (about 12,000 nodes of a structured Hexa8 mesh); larger meshes return CEOS_E_ARG.  It calls no
 * cudaMalloc or cudaFree.  The first call on a device resolves the scratch address there
 * (cudaGetSymbolAddress) and should come before any stream capture.  Calls share the scratch:
 * each clears what it uses first, and calls that overlap on the GPU race.  Synchronous;
 * returns 0, 1 (det J <= 1e-13 somewhere) or a negative CEOS_E_* code. */
int ceos_cnh_assemble_noalloc(int n_nodes, int n_elem, const double* X_device, const double* U_device,
                              const int* conn_device, const int* rowmap_device, const int* col_device,
                              long long nnz, double mu, double lambda, double* fint_device,
                              double* kval_device, void* stream);

/* ---- Device-side pieces for external materials and macro problems (no reference
 * counterpart; the reference evaluates materials inside its element loop and solves with PARDISO)
 * ---------------------------------------------------------------------------------------------- */
/* Replace the per-element parameters of a handle created with per_element materials:
 * params [n_elem][n_params] (element-major, as at creation). */
int ceos_update_params(void* handle, const double* params);
/* Deformation gradient at every Gauss point from device displacements U [3*n_nodes]:
 * F [9][8*n_elem] (row-major components, point q = gp*n_elem + e), device pointers. */
int ceos_gp_deformation_device(void* handle, const double* U_device, double* F_device, void* stream);
/* Device pointer of the committed Gauss-point state [nvars][8][ld] (FP64, or FP32 in mixed mode).
 * With model 200 (external material) each point's 27 state values are its Cauchy stress (Voigt
 * 11,22,33,12,23,13) and the 21 upper entries of its spatial tangent, read by the element loop. */
int ceos_state_device(void* handle, void** state, long long* ld, int* is_f32);
/* Write nv values per point into the committed state: q [n_pts] point ids (gp*n_elem + e),
 * vals [n_pts][nv] host arrays. */
int ceos_state_scatter(void* handle, int n_pts, const int* q, const double* vals, int nv);
/* Block-Jacobi preconditioned CG on the handle's symmetric upper CSR, on the device
 * (replaces the PARDISO solve of ModNewtonRaphsonFull.f90:44-168 for device-resident Newton):
 * solves K_ff x_f = b_f with x = 0 where fixed[i] != 0, to ||r|| <= tol ||b_f||.  K, fixed, b,
 * x are device pointers; returns 0, or CEOS_E_SOLVER when max_iter is reached. */
int ceos_pcg_create(void* handle, void** pcg);
int ceos_pcg_solve(void* pcg, const double* K_device, const unsigned char* fixed_device, const double* b_device,
                   double* x_device, double tol, int max_iter, int* iters, double* rel_res);
void ceos_pcg_destroy(void* pcg);

/* ---- Learned FE^2 surrogate (no reference counterpart) ---------------------------------------
 * MLP energy e(x), x = [(C11-1, C22-1, C33-1, C12, C23, C13)/s_C, (vf - vf0)/s_vf], width 128,
 * four softplus layers; S_k = a_k (s_W/s_C) de/dx_k (a = 2,2,2,1,1,1) and the material tangent
 * a_p a_q (s_W/s_C^2) d2e/dx_p dx_q.  Parameters: flat FP32 vector (W1 [128][7], b1, W2, b2, W3,
 * b3, W4, b4 [128][128] / [128], w5 [128], b5). */
int ceos_sur_create(int batch_max, int device, void** handle);
int ceos_sur_n_params(void);
int ceos_sur_set_params(void* handle, const float* theta);
int ceos_sur_get_params(void* handle, float* theta);
/* scales = [s_C, s_W, vf0, s_vf]; lo/hi [7]: training box of x for the range check (may be NULL). */
int ceos_sur_set_scaling(void* handle, const double* scales, const double* lo, const double* hi);
/* Gradient of L = (1/n) sum_s sw_s sum_k w_k (de/dx_k - t_k)^2 (k < 6) over one batch (n <=
 * batch_max): x [n][7], t [n][6], w [6], sw [n] (NULL: all 1) -> grad [n_params], loss.  BF16
 * tensor-core kernels, FP32 accumulation. */
int ceos_sur_gradient(void* handle, int n, const float* x, const float* t, const float* w, const float* sw,
                      float* grad, double* loss);
/* Adam training, mini-batches of `batch` from a seeded per-epoch shuffle, learning rate decaying
 * geometrically lr0 -> lr1; sample weights sw [n] or NULL; loss_hist [epochs]. */
int ceos_sur_train(void* handle, int n, const float* x, const float* t, const float* w, const float* sw, int epochs,
                   int batch, double lr0, double lr1, unsigned seed, double* loss_hist);
/* C6 [n][6], vf [n] (host) -> S [n][6], material tangent [n][36], out_of_range [n] (any may be NULL). */
int ceos_sur_evaluate(void* handle, int n, const double* C6, const double* vf, double* S, double* Cm,
                      int* out_of_range);
/* Device material step for an external-material element loop: F [9][ldF] (point q = gp*n_elem+e),
 * vf [n_elem] -> Cauchy stress and spatial tangent into state[(v*8+gp)*ld + e] (FP32 when
 * state_f32), flags [8*n_elem] = 1 outside the training box.  All device pointers. */
int ceos_sur_material_device(void* handle, int n_elem, const double* F, long long ldF, const double* vf,
                             void* state, int state_f32, long long ld, int* flags, void* stream);
/* Subtract the network's stress at C = I (tabulated over vf in [vf_lo, vf_hi]) from every later
 * stress: the undeformed state becomes stress-free, the tangent is unchanged. */
int ceos_sur_set_reference(void* handle, double vf_lo, double vf_hi);
int ceos_sur_message(void* handle, char* msg, int msg_len);
/* The 128-wide layer GEMMs of training: path 1 (the default) tcgen05 tensor cores, the four passes of
 * 128 samples in one CTA of one launch (accumulators in tensor memory), path 0 mma.sync on warps, one
 * launch per layer.  Both give the same gradient up to FP32 summation order. */
int ceos_sur_set_gemm(void* handle, int path);
void ceos_sur_destroy(void* handle);

/* ---- Batched FE^2 micro problems (no reference counterpart: CEOS solves one RVE at a time,
 * MultiScale/ModMultiscaleAnalysis.f90:445-470) ------------------------------------------------
 * n_rve periodic RVEs, RVE r a unit cube of n_cells[r]^3 Hexa8 cells with one cylindrical fibre
 * along z of volume fraction vf[r]: each cell carries the fibre's area fraction of its cross-section
 * (16 x 16 sub-points) and moduli mixed by it; both phases compressible Neo-Hookean (model 7),
 * matrix shear modulus mu_matrix, fibre modulus stiff_ratio * mu_matrix, bulk modulus
 * k_over_mu * mu in each phase. */
int ceos_fe2_create(int n_rve, const int* n_cells, const double* vf, double mu_matrix, double stiff_ratio,
                    double k_over_mu, int device, void** handle);
/* Mesh sizes and the discretised fibre fraction of every RVE (any pointer may be NULL). */
int ceos_fe2_info(void* handle, int* n_nodes, int* n_elem, int* n_red, double* vf_actual);
/* Solve every RVE under its macro deformation gradient Fbar [n_rve][9] (row-major 3x3): Newton
 * on the periodic fluctuations to ||T^T f_int|| <= tol * (its value at the start of the load
 * step), per RVE load continuation with backtracking and golden-ratio cut-back, each linear system
 * by block-Jacobi MINRES (FP32, SPD preconditioner; T^T K T may be indefinite when fibres buckle)
 * with FP64 refinement to an Eisenstat-Walker tolerance (1e-8 for the tangent).  At most
 * max_newton iterations per load step; n_cells <= 14.  Outputs the homogenized
 * first Piola stress P [n_rve][9] (row-major, the HomogenizeStress definition,
 * ModMultiscaleAnalysis.f90:140-329) and, when A != NULL, the tangent dP/dFbar [n_rve][81]
 * (row (iJ), column (kL), row-major pairs).  newton_iters / cg_iters [n_rve] may be NULL. */
int ceos_fe2_solve(void* handle, const double* Fbar, double tol, int max_newton, double* P, double* A,
                   int* newton_iters, int* cg_iters);
/* First load step of every RVE = 1/n_sub of Fbar - I (default 1: the full load at once). */
int ceos_fe2_set_increments(void* handle, int n_sub);
/* allow != 0: an RVE that cannot converge gets NaN in P and A and newton_iters -1, and
 * ceos_fe2_solve returns 2 after finishing the others (default 0: the solve fails). */
int ceos_fe2_set_allow_failures(void* handle, int allow);
/* Device-resident continuation: on != 0 (the default) runs every Newton round of a solve on the
 * device, one CUDA graph whose WHILE node repeats a round (Fbar of the trial load level, assembly,
 * failure flags, residual norms, the per-RVE accept / halve / cut-back / converge decision, vector
 * operations, the linear solve, the Newton step) until no RVE is left in Newton; the host launches it
 * once per solve.  on = 0: the host takes the per-RVE decisions between rounds (two graph launches
 * and a synchronisation per round). */
int ceos_fe2_set_device_rounds(void* handle, int on);
/* on != 0: each solve continues every RVE from the Fbar and fluctuation of its last converged
 * state (along the macro load path) instead of from Fbar = I (default 0). */
int ceos_fe2_set_warm_start(void* handle, int on);
/* RVEs the persistent solver keeps in flight (0: as many as occupancy allows). */
int ceos_fe2_set_solver_ctas(void* handle, int n);
/* mask [n_rve]: 0 leaves an RVE out of the next solves (it keeps its state and P is that of the
 * state; its rows of A are not recomputed and must not be used); NULL solves all (default). */
int ceos_fe2_set_solve_mask(void* handle, const int* mask);
/* New nominal fibre volume fractions vf [n_rve] for the same RVE sizes (cell moduli recomputed);
 * RVEs whose fraction changes restart from the undeformed state, the others keep a warm state. */
int ceos_fe2_set_fractions(void* handle, const double* vf);
/* Description of the last failure of ceos_fe2_solve (empty when none). */
/* Autotuner of the MINRES launch shape: times the first linear solve of every RVE at Fbar
 * ([n_rve][9], row-major) for threads per RVE {256, 512} x RVEs in flight {occupancy limit,
 * 2 per SM, 1 per SM}, keeps the fastest for the following solves and returns it in threads and
 * ctas (0 = occupancy limit).  ms_out[n_cand] (or NULL) receives the candidates' times (-1 for
 * duplicates).  The RVE fluctuations are unchanged.  No reference counterpart. */
int ceos_fe2_autotune(void* handle, const double* Fbar, int* threads, int* ctas, double* ms_out, int n_cand);
int ceos_fe2_message(void* handle, char* msg, int msg_len);
void ceos_fe2_destroy(void* handle);

/* ---- Host driver above the boundary (the Fortran host's role, restated in C++) ----------
 * Quasi-static analysis of one load case: QuasiStaticAnalysisFEM (ModFEMAnalysis.f90:1136-1374),
 * NewtonRaphsonFull_Solve (ModNewtonRaphsonFull.f90:44-168) and ApplyBoundaryConditionsNEW
 * (ModBoundaryConditions.f90:246-340), calling ceos_evaluate every iteration and a host
 * sparse LDL^T in place of PARDISO.  Arrays as in the reference: dofs 1-based,
 * *_init/_final item-major [n_items*n_steps]; norm_mode 0 relative, 1 absolute;
 * norm_type 2 max-abs, 1 L2.  Outputs as documented for each array. */
/* Result callback of ceos_analysis, the call sites of WriteFEMResults in QuasiStaticAnalysisFEM
 * (ModFEMAnalysis.f90:1314-1337): called once per converged substep with the analysis time,
 * the load case (1), the step (1-based among the steps of this call), the cut-back and substep
 * counters as the reference keeps them (a cut back sets SubStep = 1, a converged substep adds
 * 1), Flag_EndStep (1 when alpha = 1, the end of the step), the Newton iterations of that
 * substep and U [n_dof] (host memory, valid during the call).  A nonzero return stops the
 * analysis with CEOS_E_ABORTED. */
typedef int (*ceos_step_callback)(void* user, double time, int load_case, int step, int cutback, int substep,
                                  int flag_end_step, int n_iterations, int n_dof, const double* U);
/* Installs (cb != NULL) or removes the result callback of this handle. */
int ceos_analysis_set_callback(void* handle, ceos_step_callback cb, void* user);
/* Starting displacements of the next ceos_analysis on this handle (RestartAnalysis,
 * ModFEMAnalysis.f90:2827-2956: U of the last converged step read back from FEMAnalysis.result);
 * U0 [n_dof] is copied, NULL clears it.  The next ceos_analysis consumes it. */
int ceos_analysis_set_initial(void* handle, const double* U0);
/* Device-resident Newton for the following ceos_analysis calls on this handle (on != 0): each
 * iteration evaluates into device buffers (ceos_evaluate_device), applies the boundary conditions
 * of ApplyBoundaryConditionsNEW (ModBoundaryConditions.f90:246-340: R -= K Ubar at the first
 * iteration through the upper-symmetric product of :289-333, constrained rows and columns of K
 * zeroed with a unit diagonal, :344-536) as kernels, reduces the residual norm on the device and
 * solves K DX = -R with the device block-Jacobi PCG to the relative residual lin_tol (at most
 * lin_max_iter iterations) in place of the PARDISO solve (ModPardisoSolver.f90:343-380).  Only
 * the norm (8 bytes per iteration) and U at converged substeps return to the host; K never
 * leaves the device.  A PCG that misses lin_tol counts as a failed iteration (cut back).
 * on = 0 restores the host factorization. */
int ceos_analysis_set_device_solver(void* handle, int on, double lin_tol, int lin_max_iter);

int ceos_analysis(void* handle, int n_steps, const double* step_t0, const double* step_dt,
                  int n_fixed, const int* fixed_dofs,
                  int n_presc, const int* presc_dofs, const double* presc_init, const double* presc_final,
                  int n_force, const int* force_dofs, const double* force_init, const double* force_final,
                  double tol, int itmax, int norm_mode, int norm_type, int max_cutbacks,
                  int* iters, int* cutbacks, int n_probe, const int* probe_dofs, double* probe_out,
                  int max_log, double* norm_log, int* n_log, double* U_final);

#ifdef __cplusplus
}
#endif
#endif /* CEOS_GPU_H */
