/*
 * psp_b200 — C ABI of the B200-native sweeping-preconditioned Helmholtz solver.
 *
 * Plain pointers and sizes only; every call returns a psp_cu_status and never
 * throws.  The C++ surface (include/psp/psp.hpp) and the Python binding
 * (psp_b200/__init__.py) are thin layers over these entry points.
 *
 * Grids are natural order (x fastest, then y, then z) and complex grids carry
 * the k right-hand sides interleaved per point, i.e. the buffer layout of a
 * one-process psp::DistUniformGrid<Complex<double>> with numScalars = k
 * (PSP include/psp/dist_uniform_grid.hpp:292-342).  Complex numbers are two
 * doubles (re, im).
 *
 * Threading: a handle is thread-compatible, not thread-safe; it owns one CUDA
 * stream and all of its device memory.  The caller owns every buffer it
 * passes in.
 */
#ifndef PSP_B200_H
#define PSP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PSP_CU_OK = 0,
    PSP_CU_LOGIC_ERROR = 1,     /* std::logic_error in the reference */
    PSP_CU_RUNTIME_ERROR = 2,   /* std::runtime_error in the reference */
    PSP_CU_CUDA_ERROR = 3,
    PSP_CU_OUT_OF_MEMORY = 4,
    PSP_CU_NOT_INITIALIZED = 5,
    PSP_CU_NO_DEVICE = 6
} psp_cu_status;

typedef enum { PSP_CU_PML = 0, PSP_CU_DIRICHLET = 1 } psp_cu_boundary;

/* psp::PanelScheme (include/psp/dist_helmholtz.hpp:14-19). */
typedef enum { PSP_CU_LDL_1D = 0, PSP_CU_LDL_SELINV_1D = 1 } psp_cu_panel_scheme;

/* Arithmetic of the panel fronts and sweeps; GMRES, the residual matvec and
 * the Arnoldi/Givens work are FP64 in both modes. */
typedef enum { PSP_CU_FP64 = 0, PSP_CU_MIXED = 1 } psp_cu_precision;

/* psp::Discretization<double> (include/psp/discretization.hpp:36-110). */
typedef struct {
    double omega;
    int nx, ny, nz;
    double wx, wy, wz;
    int frontBC, rightBC, backBC, leftBC, topBC; /* psp_cu_boundary */
    int bx, by, bz;
    double sigmax, sigmay, sigmaz;
} psp_cu_disc;

typedef struct {
    int iterations;            /* GMRES inner steps taken */
    int converged;
    int lucky_breakdown;       /* B then holds the right-hand sides (solve.hpp:405-414) */
    double final_max_rel_resid;
    double solve_seconds;
    double precondition_seconds;
    double matvec_seconds;
    double arnoldi_seconds;
    int num_preconditions;
} psp_cu_stats;

typedef struct psp_cu_handle psp_cu_handle;

/* Last error message of the calling thread. */
const char* psp_cu_last_error(void);

/* DistHelmholtz<double>(disc, comm, damping, numPlanesPerPanel, cutoff)
 * (include/psp/dist_helmholtz/main.hpp:12-436).  Throws nothing; a shallow
 * domain (main.hpp:38-41) returns PSP_CU_LOGIC_ERROR. */
int psp_cu_create(const psp_cu_disc* disc, double damping, int planes_per_panel, int cutoff, int device,
                  psp_cu_handle** out);

/* ~DistHelmholtz. */
void psp_cu_destroy(psp_cu_handle* h);

/* DistHelmholtz::Initialize(velocity, panelScheme)
 * (include/psp/dist_helmholtz/initialize_finalize.hpp:12-377); velocity is a
 * host array of nx*ny*nz doubles in natural order. */
int psp_cu_initialize(psp_cu_handle* h, const double* velocity, int panel_scheme, int precision);

/* Same with the velocity already in device memory of the handle's GPU. */
int psp_cu_initialize_device(psp_cu_handle* h, const double* d_velocity, int panel_scheme, int precision);

/* Batched variants over count independent problems, one handle each (the
 * handles may live on different GPUs).  No counterpart in the reference,
 * which runs one problem per SPMD job; each element is exactly
 * psp_cu_initialize / psp_cu_solve on its own handle, run in order.  The
 * first failing element stops the batch: its status is returned and its
 * index written to *failed (-1 when every element succeeds); stats (if not
 * NULL) holds count entries. */
int psp_cu_initialize_batch(psp_cu_handle* const* h, const double* const* velocity, int count, int panel_scheme,
                            int precision, int* failed);
int psp_cu_solve_batch(psp_cu_handle* const* h, double* const* B, const int* k, int count, int m, double rel_tol,
                       psp_cu_stats* stats, int* failed);

/* DistHelmholtz::Solve(B, m, relTol) (include/psp/dist_helmholtz/solve.hpp:12-56):
 * B is a host grid of nx*ny*nz*k complex values, overwritten by the solution.
 * When the GMRES workspace of all k right-hand sides (about nx*ny*nz*k*(m+5)
 * complex doubles) does not fit in device memory, blocks of right-hand sides
 * are solved one after another, each to the tolerance; stats then report the
 * largest step count and residual over the blocks. */
int psp_cu_solve(psp_cu_handle* h, double* B, int k, int m, double rel_tol, psp_cu_stats* stats);

/* The same on a device grid owned by the caller. */
int psp_cu_solve_device(psp_cu_handle* h, double* d_B, int k, int m, double rel_tol, psp_cu_stats* stats);

/* DistHelmholtz::Finalize() (initialize_finalize.hpp:379-396): frees the factors. */
int psp_cu_finalize(psp_cu_handle* h);

/* B := A B with the global operator (Multiply, solve.hpp:613-679); host grid. */
int psp_cu_multiply(psp_cu_handle* h, double* B, int k);

/* B := M^{-1} B, one application of the sweeping preconditioner
 * (Precondition, solve.hpp:681-734); host grid. */
int psp_cu_precondition(psp_cu_handle* h, double* B, int k);

/* Device-grid variants of the two calls above. */
int psp_cu_multiply_device(psp_cu_handle* h, double* d_B, int k);
int psp_cu_precondition_device(psp_cu_handle* h, double* d_B, int k);

/* B := A B on a device grid without allocating any device memory.  No
 * counterpart in the reference: it exists for callers that cannot allocate
 * while they call -- code running inside its own CUDA stream capture, where an
 * allocation breaks the capture, and services that reserve all device memory
 * up front.  psp_cu_multiply_device allocates its nx*ny*nz*k temporary on
 * every call; this variant uses a 16 MiB file-scope device array instead, so
 * nx*ny*nz*k must not exceed 1048576 (PSP_CU_LOGIC_ERROR otherwise).  The
 * first call on a device looks up that array's device address; make it before
 * any stream capture.  All calls share the array: calls that overlap on the
 * GPU race and must be ordered by the caller.  Requires an initialized
 * handle. */
int psp_cu_multiply_device_noalloc(psp_cu_handle* h, double* d_B, int k);

/* Velocity gradient of a real misfit J(u(vel)), u = A(vel)^{-1} f:
 * d_grad[i] (+)= -Re( dA_ii/dvel_i * sum_r d_Z[i,r] d_U[i,r] ) over device
 * natural-order grids of k right-hand sides, where d_U holds the forward
 * fields and d_Z the adjoint fields A d_Z = conj(dJ/dconj(u)) (a solve with
 * the same factors, the operator being complex symmetric).  No counterpart
 * in the reference, which has no adjoint; dA_ii/dvel_i = 2 omega^2/vel_i^3 *
 * s1 s2 s3 differentiates FormGlobalRow's centre term
 * (initialize_finalize.hpp:567-568).  d_grad holds nx*ny*nz doubles;
 * accumulate != 0 adds to it.  Requires an initialized handle. */
int psp_cu_gradient_device(psp_cu_handle* h, const double* d_U, const double* d_Z, int k, double* d_grad,
                           int accumulate);

/* B := T_p B on panel p only (SolvePanel, solve.hpp:736-882); host grid. */
int psp_cu_solve_panel(psp_cu_handle* h, double* B, int k, int panel);

/* z-panel pipeline over several GPUs (the one-process form of the
 * reference's panel distribution: SubdiagonalUpdate / MultiplySuperdiagonal,
 * solve.hpp:884-948, 969-1047, and the panel-local factorizations of
 * initialize_finalize.hpp:123-322).  A rank's handle factors only panels
 * [p0, p1) (call before its first Initialize); its vectors are slabs of the
 * grid, planes z_base .. of nx*ny*k complex entries each.
 *
 * psp_cu_solve_panel_slab: SolvePanel (solve.hpp:736-882) of panel `panel`
 * on a device slab, in place.  in_mode 0: B_i := T_i B_i; 1: B_i := T_i (B_i
 * - A_{i,i-1} B_{i-1}), reading the plane below the panel; 2: B_i := T_i
 * (-A_{i,i+1} B_{i+1}), reading the plane above it; out_accumulate adds the
 * result to B_i instead of replacing it.  The slab must hold every plane the
 * solve touches: a z_base above the lowest one, or an in_mode whose
 * neighbouring panel does not exist, is a logic error; the caller makes the
 * slab reach the highest one (the library is not told the slab's length).
 *
 * psp_cu_multiply_slab: Y := A X, or Y := Bv - A X when Bv is not NULL, on
 * planes [z_first, z_first + z_count) of device slabs X, Y, Bv whose first
 * stored plane is z_slab; X must hold the planes next to that range that
 * exist in the grid (the halo): a z_slab above z_first - 1 is a logic error,
 * and the caller makes the slabs reach plane z_first + z_count. */
int psp_cu_set_panel_range(psp_cu_handle* h, int p0, int p1);
int psp_cu_solve_panel_slab(psp_cu_handle* h, double* d_B, int k, int panel, int in_mode, int out_accumulate,
                            int z_base);
int psp_cu_multiply_slab(psp_cu_handle* h, const double* d_X, double* d_Y, const double* d_Bv, int k, int z_first,
                         int z_count, int z_slab);

/* Cap on GMRES inner steps (0 = none, the reference behaviour). */
int psp_cu_set_max_iterations(psp_cu_handle* h, int max_iterations);

/* viewIterates of Solve (solve.hpp:579-585): with a basename, every GMRES
 * inner step that does not converge writes the current iterate with
 * WriteVolume (psp_cu_grid_write_volume) as <basename>-<it>, it counting
 * the inner steps from 0 across restarts (the reference's basename is
 * "iterates", relative to the working directory).  NULL turns it off. */
int psp_cu_set_view_iterates(psp_cu_handle* h, const char* basename);

/* The PRINT_RITZ_VALUES build option of the reference (solve.hpp:257-261,
 * 391-395, 422-426, 589-608) as a run-time mode: 0 off, 1 record the
 * eigenvalues of the Hessenberg matrix of the first GMRES restart cycle of
 * each right-hand side at every Solve, 2 record them and print them to
 * stdout in the reference's format.  LOGIC_ERROR for other modes. */
int psp_cu_set_ritz_values(psp_cu_handle* h, int mode);

/* The Ritz values of the last Solve that recorded them: *count per
 * right-hand side (the inner steps of its first restart cycle; 0 if none
 * were recorded) and *num_rhs; out (may be NULL) receives count*num_rhs
 * complex values, those of right-hand side r at out[2*(r*count + s)]. */
int psp_cu_get_ritz_values(const psp_cu_handle* h, int* count, int* num_rhs, double* out);

/* Host only: the eigenvalues of an n x n complex upper Hessenberg matrix H
 * (column-major, leading dimension ldh, entries below the first subdiagonal
 * ignored) into w (2n doubles), as Elemental's lapack::HessenbergEig (LAPACK
 * zhseqr, eigenvalues only) at solve.hpp:597-598 returns them.  LOGIC_ERROR
 * for bad sizes, RUNTIME_ERROR if the QR iteration does not converge or H
 * has a non-finite entry. */
int psp_cu_hessenberg_eigenvalues(int n, const double* H, int ldh, double* w);

/* Panel geometry: number of panels and, if info != NULL, 4 ints per panel
 * (lowest v, depth, padding, class) as in main.hpp:728-821. */
int psp_cu_geometry(const psp_cu_handle* h, int* num_panels, int* info);

/* The same panel geometry from a discretization alone (host only, no
 * handle or GPU): number of panels and, if info != NULL, 4 ints per panel
 * (lowest v, depth, padding, class), main.hpp:12-57, 728-821. */
int psp_cu_panel_geometry(const psp_cu_disc* disc, int planes_per_panel, int* num_panels, int* info);

/* Seconds spent in the last Initialize and bytes of stored panel factors. */
int psp_cu_setup_info(const psp_cu_handle* h, double* setup_seconds, long long* factor_bytes);

/* Factor storage after Initialize (no counterpart in the reference, whose
 * panels are always resident across its MPI ranks): the number of panels
 * whose factors stay in device memory out of num_panels, the panel
 * factorizations sweeps have rerun since Initialize for the others (each
 * recomputed panel is factored again into a per-class slot whenever a sweep
 * reaches it), and the bytes of the handle's scratch (factorization
 * transients, then the GMRES workspace).  Residency is decided at the first
 * Initialize from free device memory; PSP_B200_RESIDENT_PANELS caps it and
 * PSP_B200_SOLVE_RESERVE_RHS sets the right-hand sides whose GMRES
 * workspace is kept free (default 16). */
int psp_cu_memory_info(const psp_cu_handle* h, int* resident_panels, int* num_panels, long long* refactorizations,
                       long long* scratch_bytes);

/* Right-hand sides per GMRES block that Solve of k right-hand sides with
 * restart m would use now: k when the workspace of all of them fits beside
 * the factors, else the width of the equal blocks it solves one after
 * another (no counterpart in the reference, which holds all k at once). */
int psp_cu_solve_block_width(psp_cu_handle* h, int k, int m, int* width);

/* Host-only form of the same choice for given sizes: the GMRES block width
 * for k right-hand sides when avail_bytes of device memory are left and one
 * right-hand side's workspace takes per_rhs_bytes (cap > 0 limits it).
 * PSP_CU_OUT_OF_MEMORY, with both sizes in the message, when not even one
 * fits. */
int psp_cu_plan_block_width(int k, double avail_bytes, double per_rhs_bytes, int cap, int* width);

/* The CUDA stream (cudaStream_t) all work of the handle is issued on. */
int psp_cu_get_stream(const psp_cu_handle* h, void** stream);

/* Kernel profiling (no counterpart in the reference, which times phases with
 * mpi::Time): when on, every launch is bracketed by CUDA events on the
 * handle's stream and sweeps run without graph replay.  Categories:
 * 0 factorization GEMM, 1 panel-solve GEMM, 2 LDL diagonal blocks, 3 LDL
 * column panels, 4 front assembly, 5 extend-add, 6 solve gathers/scatters,
 * 7 stencil apply, 8 GMRES vector kernels, 9 whole sweeps. */
int psp_cu_set_profiling(psp_cu_handle* h, int on);
int psp_cu_profile_reset(psp_cu_handle* h);
int psp_cu_profile_get(psp_cu_handle* h, int category, long long* launches, double* ms, double* flops,
                       double* bytes);

/* Algorithmic flops and bytes of one sweep for k right-hand sides. */
int psp_cu_sweep_cost(const psp_cu_handle* h, int k, double* flops, double* bytes);

/* Host-only symbolic analysis (no GPU needed): the elimination tree of panel
 * class cls (0 bottom/full inner, 1 leftover, 2 top; main.hpp:705-726) as
 * 4 ints per node (ND offset, pivot count, update count, parent) in postorder,
 * and optionally its ND -> panel-natural map (nx*ny*vSize ints).  Pass
 * info = NULL to query num_nodes and vsize. */
int psp_cu_analyze_class(const psp_cu_disc* disc, int planes_per_panel, int cutoff, int cls, int* num_nodes,
                         int* vsize, int* info, int* nd_to_nat);

/* ---- grid ingest and output (psp::DistUniformGrid on one process) ------
 * A grid is nx*ny*nz points with num_scalars values per point (is_complex:
 * each value is two doubles, re and im), natural order unless stated.
 * Storage orders are the reference's GridDataOrder: 0 XYZ, 1 XZY, 2 YXZ,
 * 3 YZX, 4 ZXY, 5 ZYX (axes fastest to slowest); plane types are its
 * PlaneType: 0 XY, 1 XZ, 2 YZ. */

/* DistUniformGrid::SequentialLoad (dist_uniform_grid.hpp:349-482): reads the
 * binary file (stored in `order`) and writes the grid in natural order to
 * d_out, reordering on the current device; d_out may be device memory or
 * host memory (then staged through a temporary device buffer).
 * LOGIC_ERROR when the file cannot be opened or is shorter than the grid. */
int psp_cu_grid_load(const char* filename, int nx, int ny, int nz, int num_scalars, int is_complex, int order,
                     double* d_out);

/* DistUniformGrid::InterpolateTo (dist_uniform_grid.hpp:484-714): trilinear
 * resampling of d_in (old sizes) to d_out (new sizes) on the current device;
 * equal sizes copy.  Either may be host memory (then staged through
 * temporary device buffers).  Each value component is interpolated with the
 * reference's weights and operation order. */
int psp_cu_grid_interpolate(const double* d_in, int nx_old, int ny_old, int nz_old, int num_scalars, int is_complex,
                            double* d_out, int nx, int ny, int nz);

/* DistUniformGrid::WritePlane (dist_uniform_grid.hpp:716-1631): ASCII VTK
 * ImageData of plane `which_plane` of host grid data, one file per scalar,
 * basename_k.vti (complex: basename_k_real.vti and basename_k_imag.vti).
 * LOGIC_ERROR "Invalid plane" when the plane index is out of range. */
int psp_cu_grid_write_plane(const double* data, int nx, int ny, int nz, int num_scalars, int is_complex,
                            int plane_type, int which_plane, const char* basename);

/* DistUniformGrid::WriteVolume (dist_uniform_grid.hpp:1788-2200) for one
 * process: per scalar a basename_k.pvti description (complex: _real and
 * _imag) whose piece is basename_k/0.vti, from host grid data. */
int psp_cu_grid_write_volume(const double* data, int nx, int ny, int nz, int num_scalars, int is_complex,
                             const char* basename);

#ifdef __cplusplus
}
#endif

#endif /* PSP_B200_H */
