! ceos_gpu_mod.f90 -- ISO_C_BINDING interface of include/ceos_gpu.h for the CEOS Fortran host.
!
! The plugin type that replaces ClassFEMSystemOfEquations' EvaluateR / EvaluateKt
! (FEM/Modules/ModFEMSystemOfEquations.f90:40-93) binds these entry points; arrays are passed
! as the host holds them (real(8) U, Fint, Kg%Val; 1-based Kg%RowMap, Kg%Col, Kg%Row).
! Return codes mirror ClassStatus (Tools/ModStatus.f90:3-49): 0 success, 1 element geometry
! (det J <= 1e-13), 2 local constitutive Newton, 3 non-finite stress, negative CEOS_E_* codes.
module ceos_gpu
    use iso_c_binding
    implicit none
    private
    integer(c_int), parameter, public :: CEOS_J2_SMALL = 2, CEOS_NH_Q1P0 = 4, CEOS_SVK = 5, CEOS_CNH = 7, &
                                         CEOS_VISCO_VAR = 12, CEOS_VISCO_PRONY = 101, CEOS_J2_FINITE = 102
    integer(c_int), parameter, public :: CEOS_FP64 = 0, CEOS_MIXED = 1
    integer(c_int), parameter, public :: CEOS_E_ARG = -1, CEOS_E_CUDA = -2, CEOS_E_ALLOC = -3, CEOS_E_MESH = -4, &
                                         CEOS_E_MODEL = -5, CEOS_E_SOLVER = -6, CEOS_E_ABORTED = -7

    ! CoordX [3*n_nodes] interleaved, connectivity [8*n_elem] 1-based in the Hexa8 node order,
    ! mat_id [n_elem] 0-based into the material table (c_null_ptr: all 0)
    type, bind(C), public :: ceos_mesh
        integer(c_int) :: n_nodes, n_elem
        type(c_ptr) :: X, conn, mat_id
    end type ceos_mesh

    ! one material of the MaterialList: model id, per_element (0 shared / 1 per element), params
    type, bind(C), public :: ceos_material
        integer(c_int) :: model, per_element, n_params
        type(c_ptr) :: params
    end type ceos_material

    public :: ceos_create, ceos_pattern, ceos_evaluate, ceos_evaluate_residual, ceos_evaluate_device, &
              ceos_status, ceos_commit_state, ceos_set_committed_time, ceos_last_error, ceos_destroy

    interface
        ! AllocateKgSparseUpperTriangular (FEM/ModFEMAnalysis.f90:209-273) + material construction
        integer(c_int) function ceos_create(mesh, mats, n_mat, precision, device, h) bind(C, name="ceos_create")
            import :: c_int, c_ptr, ceos_mesh, ceos_material
            type(ceos_mesh), intent(in) :: mesh
            type(ceos_material), intent(in) :: mats(*)
            integer(c_int), value :: n_mat, precision, device
            type(c_ptr), intent(out) :: h
        end function ceos_create

        ! Kg%RowMap [3*n_nodes+1], Kg%Col [nnz], Kg%Row [nnz] (1-based, upper, sorted); any may be null
        integer(c_int) function ceos_pattern(h, n_dof, nnz, rowmap, col, row) bind(C, name="ceos_pattern")
            import :: c_int, c_long_long, c_ptr
            type(c_ptr), value :: h
            integer(c_int), intent(out) :: n_dof
            integer(c_long_long), intent(out) :: nnz
            integer(c_int) :: rowmap(*), col(*), row(*)
        end function ceos_pattern

        ! SolveConstitutiveModel + InternalForce + TangentStiffnessMatrix at U (K before the BCs)
        integer(c_int) function ceos_evaluate(h, time, U, fint, kval, n_failed) bind(C, name="ceos_evaluate")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: h
            real(c_double), value :: time
            real(c_double), intent(in) :: U(*)
            real(c_double), intent(out) :: fint(*), kval(*)
            integer(c_int), intent(out) :: n_failed
        end function ceos_evaluate

        ! the same C entry point without a tangent (EvaluateR alone): kval = c_null_ptr
        integer(c_int) function ceos_evaluate_residual(h, time, U, fint, no_kval, n_failed) &
                bind(C, name="ceos_evaluate")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: h, no_kval
            real(c_double), value :: time
            real(c_double), intent(in) :: U(*)
            real(c_double), intent(out) :: fint(*)
            integer(c_int), intent(out) :: n_failed
        end function ceos_evaluate_residual

        ! the same on device buffers and a CUDA stream (asynchronous; read the status with ceos_status)
        integer(c_int) function ceos_evaluate_device(h, time, U_d, fint_d, kval_d, stream) &
                bind(C, name="ceos_evaluate_device")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: h, U_d, fint_d, kval_d, stream
            real(c_double), value :: time
        end function ceos_evaluate_device

        integer(c_int) function ceos_status(h, n_failed) bind(C, name="ceos_status")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), intent(out) :: n_failed
        end function ceos_status

        ! SwitchConvergedState (FEM/ModFEMAnalysis.f90:1349-1353)
        integer(c_int) function ceos_commit_state(h) bind(C, name="ceos_commit_state")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function ceos_commit_state

        integer(c_int) function ceos_set_committed_time(h, t) bind(C, name="ceos_set_committed_time")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: h
            real(c_double), value :: t
        end function ceos_set_committed_time

        ! ClassStatus message and the failing element ids of ErrorElement.txt
        integer(c_int) function ceos_last_error(h, ids, max_ids, msg, msg_len) bind(C, name="ceos_last_error")
            import :: c_int, c_char, c_ptr
            type(c_ptr), value :: h
            integer(c_int) :: ids(*)
            integer(c_int), value :: max_ids, msg_len
            character(kind=c_char) :: msg(*)
        end function ceos_last_error

        subroutine ceos_destroy(h) bind(C, name="ceos_destroy")
            import :: c_ptr
            type(c_ptr), value :: h
        end subroutine ceos_destroy
    end interface
end module ceos_gpu
