/*
 * dare_gpu.h -- C ABI of the B200-native finite-volume hot path.
 *
 * Drop-in boundary for hpc-dave/dare's implicit step: Cartesian grid and
 * numbering, ghosted fields with the periodic halo fill, assembly of the
 * per-cell 7-point coefficients (DDT + diffusion + TVD convection + boundary
 * folding), and the BiCGStab(2) solve.  Every entry point is plain C: opaque
 * handles, plain pointers and sizes, int status codes (0 = OK, never aborts).
 * Host arrays passed in or out are caller-owned; device memory belongs to the
 * context.  A context is thread-compatible (one host thread at a time) and
 * issues all work on one CUDA stream.
 *
 * Citations are file:line in the hpc-dave/dare source tree.
 */
#ifndef DARE_GPU_H_
#define DARE_GPU_H_

#include <stdint.h>

#if defined(__GNUC__)
#define DARE_API __attribute__((visibility("default")))
#else
#define DARE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference throws or MPI_Aborts instead:
 *      BiCGStab2.inl:139-160, ExecutionManager.cpp:72-77) -------------------- */
#define DARE_OK 0
#define DARE_ERR_BAD_ARG (-1)
#define DARE_ERR_CUDA (-2)
#define DARE_ERR_OOM (-3)
#define DARE_ERR_STATE (-4)
#define DARE_ERR_UNSUPPORTED (-5)
#define DARE_ERR_TIMEOUT (-6)       /* a bounded device wait ran out (the call returned; the context stays usable) */

/* ---- neighbour slots: CartesianNeighbor (Grid/Cartesian/CartesianMesh.h:67-77) */
#define DARE_CENTER 0
#define DARE_WEST 1
#define DARE_EAST 2
#define DARE_SOUTH 3
#define DARE_NORTH 4
#define DARE_BOTTOM 5
#define DARE_TOP 6

/* ---- boundary conditions folded into boundary rows
 *      (test/Verification/counter_diffusion1D.cpp:123-146) ------------------- */
#define DARE_BC_PERIODIC 0
#define DARE_BC_DIRICHLET 1
#define DARE_BC_NEUMANN 2

/* ---- flux limiters: Equations/FluxLimiter.h:41-173 (+ van Leer, new) ------ */
#define DARE_LIMITER_CDS 0
#define DARE_LIMITER_UPWIND 1
#define DARE_LIMITER_VANALBADA 2
#define DARE_LIMITER_MINMOD 3
#define DARE_LIMITER_VANLEER 4

/* ---- time schemes of the Divergence operators ------------------------------
 * Equations/TimeDiscretizationSchemes.h:29-76, weights w[0..T]: the implicit
 * coefficients of div(...) are scaled by w[0], and each explicit level t >= 1
 * adds w[t] * A * (rhs_E - rhs_W + ...) of the operator's face stencil
 * (Grid/Cartesian/Divergence_Cartesian.inl:186-205; the levels are copies of
 * the level-0 stencil, :61-62).  DDT keeps its implicit weights (1, 1). */
#define DARE_SCHEME_EULER_BACKWARD 0  /* (1) */
#define DARE_SCHEME_EULER_FORWARD 1   /* (0, 1) */
#define DARE_SCHEME_CRANK_NICHOLSON 2 /* (0.5, 0.5) */
#define DARE_SCHEME_ADAMS_BASHFORTH 3 /* (0, 1.5, -0.5) */
#define DARE_SCHEME_ADAMS_MOULTON 4   /* (5/12, 8/12, -1/12) */

/* ---- preconditioners (right, TrilinosSolver.inl:84-85) --------------------- */
#define DARE_PREC_NONE 0
#define DARE_PREC_JACOBI 1

/* ---- solver precision modes ------------------------------------------------ */
#define DARE_PRECISION_FP64 0
#define DARE_PRECISION_FP32_REFINE 1

/* ---- solve status (BiCGStab2.inl:322-571) ---------------------------------- */
#define DARE_SOLVE_CONVERGED 0
#define DARE_SOLVE_MAXIT 1
#define DARE_SOLVE_BREAKDOWN 2   /* breakdown_step holds the reference step 3/4/7/14/20/21 */
#define DARE_SOLVE_NAN 3

typedef struct dare_ctx dare_ctx;
typedef struct dare_grid dare_grid;
typedef struct dare_field dare_field;
typedef struct dare_system dare_system;

typedef struct {
    int dim;
    int num_ghost;
    int64_t n[3];              /* internal cells per dimension (1 when inactive) */
    int64_t n_ghosted[3];      /* incl. ghost layers in active dimensions */
    int64_t num_cells;         /* internal */
    int64_t num_cells_ghosted;
    double dx[3];
    double volume;
    double area[3];
    int periodic[3];
    int staggered[3];          /* staggered representation (dare_grid_create_staggered) */
    double origin[3];          /* position of the lower face of internal cell 0 (-dx/2 when staggered) */
} dare_grid_info;

/* Assembly description: the composed user functor of the reference's time
 * loops,
 *     mb  = ddt(field);  mb += div(TVD(vel) * field);  mb -= div(D, grad(mb));
 *     then Dirichlet / Neumann folding on non-periodic faces (W,E,S,N,B,T),
 * replacing Trilinos<SC>::Build(grep, field, functor) (MatrixSystem/Trilinos.h:107-111).
 * Face arrays live in device memory with the staggered face layout
 *     x-faces (nx+1, ny, nz), y-faces (nx, ny+1, nz), z-faces (nx, ny, nz+1),
 * entry [i][j][k] of the x-faces being the face between cells i-1 and i. */
typedef struct {
    double dt;                       /* > 0: implicit-Euler DDT (DDT.inl:39-81) */
    int diffusion;                   /* 0 none, 1 scalar D, 2 face arrays */
    double D;
    const double* face_D[3];
    int convection;                  /* 0 none, 1 constant velocity, 2 face velocity arrays */
    int limiter;                     /* DARE_LIMITER_* */
    double vel[3];
    const double* face_vel[3];
    int scheme;                      /* DARE_SCHEME_*, time scheme of both div(...) terms */
} dare_assembly_desc;

/* One term of a composed assembly functor: the MatrixBlock expressions of a
 * user functor for Trilinos<SC>::Build (MatrixSystem/Trilinos.h:107-111),
 *     (*mblock) = ddt(field);                  DDT, DARE_OP_SET
 *     (*mblock) -= div(grad(*mblock));         DIFFUSION with D = 1, DARE_OP_SUB
 *     mblock->Add(n, div(u * field).GetSlice(n));   CONVECTION for component n, DARE_OP_ADD
 * (MatrixBlock_Cartesian.inl:480-593; counter_diffusion1D.cpp:107-148,
 * advection_periodic2D.cpp:108-126).  The terms apply in order to every
 * component (component = -1) or to one; SET starts a component's block
 * afresh, ADD and SUB add the term or its negative.  After the last term the
 * non-periodic faces are folded with each component's conditions
 * (dare_system_set_bc, dare_system_set_bc_component).  Face arrays as in
 * dare_assembly_desc.  COEFFS is any other expression of a functor,
 * evaluated by the caller on the device: per-cell values of the 7 slots
 * (CENTER, WEST, EAST, SOUTH, NORTH, BOTTOM, TOP; NULL slots are 0) and of the
 * right-hand side, each an array over one component's internal cells, set,
 * added or subtracted like the other terms (and folded with them at the end). */
enum { DARE_TERM_DDT = 0, DARE_TERM_DIFFUSION = 1, DARE_TERM_CONVECTION = 2, DARE_TERM_COEFFS = 3 };
enum { DARE_OP_SET = 0, DARE_OP_ADD = 1, DARE_OP_SUB = 2 };
typedef struct {
    int kind;                        /* DARE_TERM_* */
    int op;                          /* DARE_OP_* */
    int component;                   /* -1: every component; else that component only */
    double dt;                       /* DDT: time step (> 0) */
    double D;                        /* DIFFUSION: div(D grad(mb)); 1 for div(grad(mb)) */
    const double* face_D[3];         /* DIFFUSION: face diffusivities instead of D (all three or none) */
    double vel[3];                   /* CONVECTION: constant velocity ... */
    const double* face_vel[3];       /* ... or face velocities (all three or none) */
    int limiter;                     /* CONVECTION: DARE_LIMITER_* */
    int scheme;                      /* DIFFUSION / CONVECTION: DARE_SCHEME_* of the div(...) */
    const double* coef[7];           /* COEFFS: device arrays of the 7 slots (NULL: 0) ... */
    const double* coef_rhs;          /* ... and of the right-hand side (NULL: 0) */
} dare_term;

typedef struct {
    double tol;             /* ABSOLUTE tolerance on ||r||_2 (stop criterion RNORM,
                               BiCGStab2.inl:34,561-565); tol_abs = rel * ||b|| for a relative one */
    int max_it;             /* "Maximum Iterations" */
    int precond;            /* DARE_PREC_NONE / DARE_PREC_JACOBI */
    int precision;          /* DARE_PRECISION_FP64 / DARE_PRECISION_FP32_REFINE */
    double inner_rel_tol;   /* FP32 inner solve: relative reduction per refinement (e.g. 1e-5) */
    int inner_max_it;       /* FP32 inner solve iteration cap per refinement */
    int max_refinements;
    int check_every;        /* iteration pairs between host status polls (0 = by grid size) */
    int compute_true_residual; /* report ||b - A x||_2 in FP64 after the solve */
    int tol_relative;       /* 1: stop on ||r|| <= tol * ||b||_2 (||b|| computed on the device) */
} dare_solver_params;

typedef struct {
    int iters;              /* reference num_iteration (k) */
    int converged;
    int status;             /* DARE_SOLVE_* */
    int breakdown_step;
    double res_abs;         /* last recurrence residual check (reference norm_residual) */
    double true_res_abs;    /* ||b - A x||_2, FP64 (if requested) */
    double b_norm;          /* ||b||_2 */
    int refinements;        /* FP32_REFINE: outer FP64 corrections */
    int inner_iters;        /* FP32_REFINE: total inner iterations */
    int fallback_used;      /* FP32_REFINE: fell back to the FP64 solve */
    double tol_abs;         /* absolute tolerance that was applied */
} dare_solve_report;

/* ---- context --------------------------------------------------------------- */
DARE_API int dare_ctx_create(int device, dare_ctx** out);
DARE_API int dare_ctx_destroy(dare_ctx* ctx);
/* Use an external cudaStream_t (NULL restores the context's own stream). */
DARE_API int dare_ctx_set_stream(dare_ctx* ctx, void* stream);
DARE_API void* dare_ctx_get_stream(dare_ctx* ctx);
DARE_API int dare_ctx_synchronize(dare_ctx* ctx);
DARE_API const char* dare_ctx_last_error(const dare_ctx* ctx);
/* Kernel launches this context issued since creation (for launch accounting). */
DARE_API int64_t dare_ctx_launch_count(const dare_ctx* ctx);
/* Optional per-kernel CUDA-event timing on the context's stream (no reference
 * counterpart: the reference has no timers).  Kernel ids: 0 assembly,
 * 3..7 the five fused BiCGStab(2) kernels (steps 5-7, 8-11, 12-14, 15-23, 24-25). */
DARE_API int dare_ctx_set_profiling(dare_ctx* ctx, int on);
DARE_API int dare_ctx_reset_kernel_stats(dare_ctx* ctx);
DARE_API int dare_ctx_kernel_stats(const dare_ctx* ctx, int kernel_id, double* total_ms, int64_t* count);
/* Wall time of the work issued on the context's stream between start and stop,
 * from CUDA events (stop synchronizes). */
DARE_API int dare_ctx_timer_start(dare_ctx* ctx);
DARE_API int dare_ctx_timer_stop(dare_ctx* ctx, double* ms);

/* ---- grid: Cartesian<Dim> + CartesianRepresentation (np = 1)
 *      Grid/Cartesian/CartesianMesh.inl:33-112, CartesianRepresentation.inl:31-227 */
DARE_API int dare_grid_create(dare_ctx* ctx, int dim, const int64_t n[3], const double size[3],
                     int num_ghost, const int periodic[3], dare_grid** out);
/* A staggered representation, grid->GetRepresentation(Options)
 * (CartesianRepresentation.inl:33-76): n[] and size[] describe the base grid;
 * along every direction with staggered[d] != 0 that is not periodic the
 * representation has n[d] + 1 cells of the base width size[d] / n[d], the
 * first one centred on the base grid's lower face (origin -dx/2).  Fields,
 * systems and solves on it work as on any grid. */
DARE_API int dare_grid_create_staggered(dare_ctx* ctx, int dim, const int64_t n[3], const double size[3],
                                        int num_ghost, const int periodic[3], const int staggered[3],
                                        dare_grid** out);
DARE_API int dare_grid_destroy(dare_grid* g);
DARE_API int dare_grid_get_info(const dare_grid* g, dare_grid_info* info);

/* ---- field: Field<Grid,SC,1> time levels of ghosted GridVectors
 *      Data/Field.h:47-138, Data/GridVector.h:42-251 (level 0 = new, 1 = old) */
DARE_API int dare_field_create(dare_grid* g, int num_levels, dare_field** out);
/* Field<Grid,SC,N> with N = num_components (1..64): host arrays of upload and
 * download interleave the components, ghosted[cell * N + c]
 * (Data/GridVector.inl:68-71); halo exchange and copy-to-old act on every component. */
DARE_API int dare_field_create_n(dare_grid* g, int num_levels, int num_components, dare_field** out);
DARE_API int dare_field_num_components(const dare_field* f);
DARE_API int dare_field_destroy(dare_field* f);
DARE_API int dare_field_upload(dare_field* f, int level, const double* host_ghosted);
DARE_API int dare_field_download(dare_field* f, int level, double* host_ghosted);
DARE_API double* dare_field_device_ptr(dare_field* f, int level);
/* Field::ExchangeHaloCells (Field.inl:100-103): periodic face ghosts of level 0 */
DARE_API int dare_field_exchange_halo(dare_field* f);
/* Field::CopyDataVectorsToOldTimeStep (Field.inl:88-93) */
DARE_API int dare_field_copy_to_old(dare_field* f);

/* ---- field output: io::VTKWriter<Cartesian<Dim>>(exman, time, step).Write(base_path, &vec...)
 *      (IO/VTKWriter.h:73-160, IO/VTKWriter.inl:34-86) for one grid on one rank.
 *      Writes <base_path>/<grid_name>_<step>.pvts and the piece
 *      <base_path>/<grid_name>_<step>/<grid_name>_<step>_0.vts: the ghosted grid
 *      (Grid/Cartesian/VTKOptions_Cartesian.h:146-323), one Float64 cell array per
 *      field named names[f], "TimeValue" when time >= 0.  base_path and the
 *      subdirectory are created when missing (one level each). */
DARE_API int dare_vtk_write(dare_field* const* fields, int level, const char* const* names, int count,
                            const char* base_path, const char* grid_name, int step, double time);
/* The same from host arrays over the ghosted grid (num_ghost layers on each
 * active side, the grid's numbering with the last dimension fastest); needs no GPU. */
DARE_API int dare_vtk_write_host(int dim, const int64_t n[3], const double size[3], int num_ghost,
                                 const double* const* data, const char* const* names, int count,
                                 const char* base_path, const char* grid_name, int step, double time);

/* ---- linear system: the structured 7-diagonal form of Trilinos<SC>'s A, x, B
 *      (MatrixSystem/Trilinos.h:51-314) -------------------------------------- */
DARE_API int dare_system_create(dare_grid* g, dare_system** out);
/* MatrixBlock<Cartesian<Dim>,GO,SC,N>: one 7-point stencil per component, no
 * coupling between components (Grid/Cartesian/MatrixBlock_Cartesian.h); rows
 * and columns interleave the components, row = cell * N + c, column =
 * neighbour * N + c (MatrixBlock_Cartesian.inl:127-240), in the host arrays of
 * set/get_coefficients ([7][ncell * N]), the initial guess, the solution and
 * the CSR export.  Assembly applies the descriptor to each component of an
 * N-component field; one BiCGStab2 iteration runs on all components together
 * (the reference solves the whole row map). */
DARE_API int dare_system_create_n(dare_grid* g, int num_components, dare_system** out);
DARE_API int dare_system_num_components(const dare_system* s);
DARE_API int dare_system_destroy(dare_system* s);
/* face: DARE_WEST..DARE_TOP; non-periodic faces need DIRICHLET or NEUMANN */
DARE_API int dare_system_set_bc(dare_system* s, int face, int type, double value);
/* The condition of one field component on one face (component -1: every
 * component, as dare_system_set_bc).  A functor that folds the components
 * differently, e.g. counter_diffusion1D.cpp:123-146 (Dirichlet for component 0
 * and Neumann for component 1 on the west face, the reverse on the east). */
DARE_API int dare_system_set_bc_component(dare_system* s, int component, int face, int type, double value);
/* Trilinos<SC>::Build -> BuildNew (Trilinos.inl:48-60,285-385) with the fused
 * functor above; x0 = field level 0 (the initial guess). DDT reads level 1 when
 * the field has 2+ levels, else level 0; convection reads level 0. */
DARE_API int dare_assemble(dare_system* s, const dare_assembly_desc* desc, dare_field* field);
/* Trilinos<SC>::Build with a composed functor given as `nterms` terms (see
 * dare_term); x0 = field level 0.  DDT reads level 1 when the field has 2+
 * levels; convection reads level 0. */
DARE_API int dare_assemble_terms(dare_system* s, const dare_term* terms, int nterms, dare_field* field);
/* Replace coefficients with user-built MatrixBlocks (host SoA: diag[7][ncells]
 * in slot order CENTER..TOP, removed entries 0), rhs and initial guess. */
DARE_API int dare_system_set_coefficients(dare_system* s, const double* diag7, const double* rhs,
                                 const double* x0);
DARE_API int dare_system_get_coefficients(dare_system* s, double* diag7, double* rhs);
DARE_API int dare_system_set_initial_guess(dare_system* s, const double* x0);
DARE_API int dare_system_get_solution(dare_system* s, double* x);
DARE_API double* dare_system_device_ptr(dare_system* s, int which); /* 0..6 diag, 7 rhs, 8 x */
/* CSR export for parity (MatrixBlock::Finalize, MatrixBlock_Cartesian.inl:127-240;
 * rows sorted by column as Tpetra fillComplete / Trilinos::PrintRow, Trilinos.inl:185-212) */
DARE_API int64_t dare_system_csr_nnz(dare_system* s);
DARE_API int dare_system_export_csr(dare_system* s, int64_t* rowptr, int64_t* cols, double* vals);
/* Trilinos::CopyTo (Trilinos.inl:166-177): solution into field level 0 */
DARE_API int dare_system_copy_to(dare_system* s, dare_field* f);

/* ---- solve: TrilinosSolver::Solve(BumbleBee, "BICGSTAB2", M, A, x, B, p)
 *      (TrilinosSolver.inl:69-93) -> BiCGStab2::Solve (BiCGStab2.inl:166-582) */
DARE_API void dare_solver_params_default(dare_solver_params* p);
DARE_API int dare_bicgstab2_solve(dare_system* s, const dare_solver_params* p, dare_solve_report* rep);

/* One implicit time step of the reference's driver loop
 * (test/Verification/counter_diffusion1D.cpp:170-217): Build, Solve, CopyTo,
 * ExchangeHaloCells, CopyDataVectorsToOldTimeStep. */
DARE_API int dare_timestep(dare_system* s, dare_field* f, const dare_assembly_desc* desc,
                  const dare_solver_params* p, dare_solve_report* rep);
/* nsteps such steps of a field kept in host memory: before each step the
 * field (level 0, and level 1 from it) is read from `host`, after it the
 * result is written back to `host`.  `host`: pinned, the field's device
 * layout (component-major ghosted levels; for one component the ghosted
 * layout).  The download of one step's result and the upload of the next
 * step's input are pipelined in slices on two streams (PCIe carries both
 * directions at once); every step moves the whole field both ways.  On
 * single-component 3-D grids the Build of a step runs while its input is
 * still arriving, slice by slice; the results equal the loop of single
 * calls bit for bit, and after the last step level 1 equals level 0.
 * reps: nsteps reports, or NULL.  Returns with the last result in `host`. */
DARE_API int dare_timesteps_host(dare_system* s, dare_field* f, const dare_assembly_desc* desc,
                                 const dare_solver_params* p, int nsteps, double* host, dare_solve_report* reps);

/* ---- slabs of i-planes: the grid distributed as the reference distributes
 *      it over ranks (Grid/Cartesian/CartesianDistribution.h:94-380,
 *      MPI/HaloBuffer.inl:30-208, Tpetra's sum over ranks in every dot of
 *      BiCGStab2.inl:339-559), all slabs on the system's device.
 * Slab s owns planes [i0, i1) (n0 split into runs, the first n0 % S one
 * plane longer) with its own field (every time level, ghosted), system rows
 * and solver vectors.  Before an assembly num_ghost boundary planes of the
 * field cross to each x neighbour; before every SpMV one boundary plane of
 * the operand (of every field component); every dot product sums all
 * slabs' partials.  FP64 solves (plain or Jacobi), 1 to 8 slabs of at least
 * max(num_ghost, 2) planes.  The slabs inherit the system's grid, field
 * components and face conditions (per component too); x faces shared by two
 * slabs (every x face of a periodic x) stay unfolded. */
typedef struct dare_slabs dare_slabs;
DARE_API int dare_slabs_create(dare_system* s, int num_slabs, int num_levels, dare_slabs** out);
DARE_API int dare_slabs_destroy(dare_slabs* sl);
DARE_API int dare_slabs_count(const dare_slabs* sl);
DARE_API int dare_slabs_range(const dare_slabs* sl, int slab, int64_t* i0, int64_t* i1);
/* The slab's own system and field (owned by the slabs; read and write them
 * with the dare_system_* / dare_field_* calls, do not destroy them).  Solve
 * the slabs together with dare_slabs_solve: a slab's system solved on its own
 * sees zeros beyond its first and last plane. */
DARE_API dare_system* dare_slabs_system(dare_slabs* sl, int slab);
DARE_API dare_field* dare_slabs_field(dare_slabs* sl, int slab);
DARE_API int dare_slabs_set_bc(dare_slabs* sl, int face, int type, double value);
/* Every level of a field of the system's grid into the slabs (each slab its
 * planes and num_ghost planes either side) / the slabs back into it. */
DARE_API int dare_slabs_scatter(dare_slabs* sl, dare_field* f);
DARE_API int dare_slabs_gather(dare_slabs* sl, dare_field* f);
/* Field::ExchangeHaloCells: periodic j / k ghosts in each slab, then the x
 * ghost planes from the neighbouring slabs (wrapping on a periodic x). */
DARE_API int dare_slabs_exchange_halo(dare_slabs* sl);
DARE_API int dare_slabs_copy_to_old(dare_slabs* sl);
/* Trilinos::Build on every slab; descs[s] describes slab s, its face arrays
 * covering its own planes (n_s + 1 x faces: global faces i0 .. i1, face 0
 * for the last one on a periodic x; the slab's planes of the y and z faces). */
DARE_API int dare_slabs_assemble(dare_slabs* sl, const dare_assembly_desc* descs);
DARE_API int dare_slabs_solve(dare_slabs* sl, const dare_solver_params* p, dare_solve_report* rep);
DARE_API int dare_slabs_copy_to(dare_slabs* sl);
/* Build, Solve, CopyTo, ExchangeHaloCells, CopyDataVectorsToOldTimeStep */
DARE_API int dare_slabs_timestep(dare_slabs* sl, const dare_assembly_desc* descs, const dare_solver_params* p,
                                 dare_solve_report* rep);

/* Face diffusivity as the linear interpolation of cell values to faces
 * (Interpolation_Cartesian.h:139-158: (D_lo + D_hi) * 1/2, periodic wrap on
 * periodic faces, boundary faces take the adjacent cell value).
 * cell_D: device, internal cells; face_D[d]: device, face layout above. */
DARE_API int dare_face_average(dare_grid* g, const double* cell_D, double* face_D[3]);

/* ---- batched uneven solves -------------------------------------------------
 * Many independent 3D boxes, each one implicit-Euler diffusion step
 * (DDT + div(D grad), Dirichlet/Neumann folding per face: the functor of
 * test/Verification/counter_diffusion1D.cpp:113-146 in 3D), each solved by
 * Jacobi-BiCGStab(2) (BiCGStab2.inl:166-582) with its own tolerance check and
 * status, all in one persistent launch.  Fields are internal cells,
 * ordinal (i*ny + j)*nz + k; the field is the initial guess and phi_old. */
typedef struct {
    int64_t n[3];          /* cells per dimension (>= 3 each) */
    double size[3];        /* box lengths */
    double D;              /* constant diffusivity */
    double dt;             /* implicit Euler step */
    int bc_type[6];        /* W,E,S,N,B,T: DARE_BC_DIRICHLET or DARE_BC_NEUMANN */
    double bc_value[6];
} dare_batch_instance;

typedef struct {
    int iters;
    int converged;
    int status;            /* DARE_SOLVE_* */
    int breakdown_step;
    double res_abs;        /* last recurrence residual (or true residual after a tau = 0 exit) */
    double b_norm;
    double tol_abs;
} dare_batch_report;

typedef struct dare_batch dare_batch;
DARE_API int dare_batch_create(dare_ctx* ctx, int count, const dare_batch_instance* inst, dare_batch** out);
DARE_API int dare_batch_destroy(dare_batch* bt);
DARE_API int64_t dare_batch_num_cells(const dare_batch* bt, int idx);
DARE_API int dare_batch_set_field(dare_batch* bt, int idx, const double* host_phi);
DARE_API int dare_batch_get_field(dare_batch* bt, int idx, double* host_phi);
/* Set every instance's field to 0 on the device (phi_0 = 0 start). */
DARE_API int dare_batch_zero_fields(dare_batch* bt);
/* Solves every instance (p: tol, tol_relative, max_it; Jacobi, FP64). The
 * fields are replaced by the solutions; reports (host, count entries) may be NULL. */
DARE_API int dare_batch_solve(dare_batch* bt, const dare_solver_params* p, dare_batch_report* reports);
/* Picks the block size and the cells each thread handles per sweep (per size
 * class) by timing solves of the current fields, which are restored. */
DARE_API int dare_batch_autotune(dare_batch* bt, const dare_solver_params* p, int* chosen_block);
DARE_API int dare_batch_get_tuning(const dare_batch* bt, int* block, int vec_by_size[8]);

/* ---- residual norm without device allocation -------------------------------
 * No counterpart in the reference (DaRe computes residuals inside Tpetra).
 * ||b - A x||_2 of a structured 7-point system of ONE field component given
 * as plain device arrays (diag7: 7 x ncells in slot order CENTER..TOP, x, b
 * over internal cells, ordinal (i*ny + j)*nz + k; neighbours past a
 * non-periodic face are ignored).  Systems with several components per cell
 * are not supported here (their slots interleave the components).  The result is
 * written as one double to the device pointer norm_out, on `stream` (a
 * cudaStream_t, NULL = legacy default stream).  It is for callers that cannot
 * call cudaMalloc mid-run -- host codes whose device memory is owned by their
 * own allocator or budget, or that must not stall other streams with the
 * device synchronization cudaMalloc implies: it allocates nothing and keeps
 * its scratch (4096 partial sums plus counters, about 33 KB per device) in a
 * fixed device array held until process exit.  Grids whose (j,k) plane needs
 * more than 4096 tiles of 32 x 8 cells (ny*nz above about 1M) are rejected
 * with DARE_ERR_UNSUPPORTED and a message in `err` (may be NULL).  All calls
 * on a device share that array: calls that overlap on the GPU race and must
 * be serialized by the caller.  The first call on a device looks up the
 * array's device address and keeps it for the life of the process, so make
 * that call before capturing any stream there, and do not call it again on a
 * device after cudaDeviceReset (the array's address may change). */
DARE_API int dare_residual_norm_noalloc(int dim, const int64_t n[3], const int periodic[3], const double* diag7,
                                        const double* x, const double* b, double* norm_out, void* stream,
                                        char* err, int err_len);

/* ---- learned linear preconditioner ---------------------------------------------
 * No counterpart in the reference: DaRe preconditions BiCGStab2 with Jacobi
 * only (BiCGStab2.inl:258-261, 568-571).  This is the preconditioner of
 * the Jacobi-folded system Ahat = A D^-1:
 *     N(u) = u + U(u),
 * U a bias-free, activation-free (so linear) convolutional U-Net on one 3D
 * grid whose three sizes are multiples of 8: four levels of 16, 32, 64, 64
 * channels, 3x3x3 kernels with zero padding, 2x2x2 average-pool restriction,
 * nearest-neighbour prolongation added to the encoder output of the finer
 * level (additive skip).  Eight convolutions: enc0 1->16, enc1 16->32,
 * enc2 32->64, enc3 64->64, dec3 64->64, dec2 64->32, dec1 32->16,
 * dec0 16->1.  Weights and activations are BF16, accumulation FP32 (tcgen05
 * tensor memory).  Vectors are FP32 over the internal cells, ordinal
 * (i*ny + j)*nz + k, in device memory.  Parameters are FP32 master weights,
 * layer after layer, each [27][cout][cin] with tap t = (di+1)*9 + (dj+1)*3 +
 * (dk+1) reading input cell (i+di, j+dj, k+dk). */
typedef struct dare_unet dare_unet;

typedef struct {
    float lr;                /* Adam step size */
    float beta1, beta2, eps; /* Adam moments */
    int batch;               /* (residual, error) pairs per optimiser step */
    int steps;               /* optimiser steps per dare_unet_train_on_system call */
    int max_pairs_per_rhs;   /* solver iterates turned into pairs per call */
    uint64_t seed;           /* minibatch sampling */
} dare_unet_train_params;

typedef struct {
    int pairs_added;         /* pairs generated from the plain solver by this call */
    int pairs_total;         /* pairs held in the training ring */
    int plain_iters;         /* iterations of the plain solve to the tolerance */
    int steps;               /* optimiser steps taken */
    double loss_first;       /* mean relative squared error of the first / last step */
    double loss_last;
} dare_unet_train_report;

typedef struct {
    int iteration_budget;    /* learned inner iterations allowed in total before the
                                automatic switch to the plain FP64 Jacobi-BiCGStab2 */
    int inner_max_it;        /* per refinement */
    double inner_rel_tol;    /* relative reduction of each inner solve */
    int max_refinements;
} dare_learned_params;

DARE_API void dare_unet_train_params_default(dare_unet_train_params* p);
DARE_API void dare_learned_params_default(dare_learned_params* p);
/* Randomly initialised network (He-style scale, dec0 starts at zero so N = I). */
DARE_API int dare_unet_create(dare_ctx* ctx, const int n[3], uint64_t seed, dare_unet** out);
/* The coarse-correction form for systems on the grid n_fine (sizes multiples
 * of 16): the same U-Net runs on the 2x restricted grid n_fine / 2,
 *     N(u) = u + P U(R u),
 * R the mean of the 8 children of a coarse cell, P the nearest prolongation
 * (every fine cell receives its parent's value), so no convolution runs at
 * the system's resolution.  dare_unet_apply and dare_bicgstab2_learned take
 * vectors of the system's grid; dare_unet_train_on_system stores the
 * restrictions (R r, R e) of the solver's pairs (the fine loss
 * ||r + P U(R r) - e||^2 equals 8 ||R r + U(R r) - R e||^2 plus a term
 * without U); dare_unet_loss_grad / dare_unet_train_step and
 * dare_unet_read_activation work on the network's (coarse) grid.  Weights
 * are interchangeable with a full-resolution network of the same layers.
 * No counterpart in the reference. */
DARE_API int dare_unet_create_coarse(dare_ctx* ctx, const int n_fine[3], uint64_t seed, dare_unet** out);
/* The system grid a network preconditions (n_fine of a coarse-form network,
 * else its own grid); returns 1 for the coarse form, 0 for the
 * full-resolution form, < 0 on a bad argument.  No reference counterpart. */
DARE_API int dare_unet_system_shape(const dare_unet* net, int n[3]);
DARE_API int dare_unet_destroy(dare_unet* net);
/* Polls after which a bounded wait between the roles of a tensor-core
 * convolution CTA (producer, MMA issuer, epilogue) gives up: the CTA raises
 * its abort flag, waits for its own MMAs and copies in flight, frees its
 * tensor memory and returns; the call then reports DARE_ERR_TIMEOUT and the
 * network stays usable.  0 restores the default (2^22 polls).  No reference
 * counterpart. */
DARE_API int dare_unet_set_wait_limit(dare_unet* net, int64_t polls);
/* Test hook for that failure path: in the next forward convolution of 16 or
 * more input channels, the first CTA's producer leaves its first input plane
 * unstaged (no arrive, no copies), so that CTA's bounded waits run out.  One
 * shot.  No reference counterpart. */
DARE_API int dare_unet_debug_skip_plane(dare_unet* net);
DARE_API int64_t dare_unet_num_params(const dare_unet* net);
DARE_API int dare_unet_get_weights(dare_unet* net, float* host, int64_t count);
DARE_API int dare_unet_set_weights(dare_unet* net, const float* host, int64_t count);
/* z = N(u) (device vectors on the system's grid, may not alias). */
DARE_API int dare_unet_apply(dare_unet* net, const float* u, float* z);
/* Loss over `count` pairs stored back to back (r[c*ncell..], e[c*ncell..]):
 * mean over pairs of ||N(r) - e||^2 / ||e||^2; its gradient with respect to
 * every parameter is written to grad_host (num_params floats, may be NULL). */
DARE_API int dare_unet_loss_grad(dare_unet* net, const float* r, const float* e, int count, double* loss,
                                 float* grad_host);
/* One Adam step on the mean loss of `count` device pairs. */
DARE_API int dare_unet_train_step(dare_unet* net, const float* r, const float* e, int count,
                                  const dare_unet_train_params* p, double* loss);
/* Solve the assembled system with the plain FP64 Jacobi-BiCGStab2 from its
 * current x to ||b - A x|| <= tol ||b||, turn the solver's iterates x_k into pairs (r_k = b - A x_k,
 * e_k = D (x* - x_k), D the diagonal), add them to the training ring and take
 * p->steps optimiser steps on minibatches drawn from the ring.  On return the
 * system holds the converged plain solution x*. */
DARE_API int dare_unet_train_on_system(dare_unet* net, dare_system* s, double tol, const dare_unet_train_params* p,
                                       dare_unet_train_report* rep);
/* Number of optimiser steps and pairs seen since creation. */
DARE_API int dare_unet_stats(const dare_unet* net, int64_t* steps, int64_t* pairs_seen);
/* Launch shape of a convolution kernel after its first launch: layer 0..7
 * (enc0..dec0 as above), kind 0 forward, 1 data gradient, 2 weight gradient;
 * info = {grid x, grid y, grid z, dynamic smem bytes, planes per CTA, taps
 * per CTA (weight gradient) or staged-plane ring depth (the others), TMEM
 * columns, resident CTAs per SM}.  DARE_ERR_STATE before the first launch. */
DARE_API int dare_unet_launch_info(const dare_unet* net, int layer, int kind, int64_t info[8]);
/* Internal activation `which` (0 S0, 1 P1, 2 S1, 3 P2, 4 S2, 5 P3, 6 E3) as
 * FP32 [cell][channel] over the internal cells of its level. */
DARE_API int dare_unet_read_activation(dare_unet* net, int which, float* host, int64_t count);

/* Mixed-precision BiCGStab2 with the learned preconditioner: FP64 iterative
 * refinement r = b - A x, an FP32 inner BiCGStab2 on Ahat N y = r with FP64
 * dot products, x += D^-1 N y.  When the learned phase misses the stated
 * iteration budget (or stops contracting) the plain FP64 Jacobi-BiCGStab2
 * continues from the current iterate; rep->fallback_used reports that.  The
 * final residual is the FP64 ||b - A x||_2.  p->tol / tol_relative set the
 * stop test, p->max_it caps the fallback. */
DARE_API int dare_bicgstab2_learned(dare_system* s, dare_unet* net, const dare_solver_params* p,
                                    const dare_learned_params* lp, dare_solve_report* rep);

#ifdef __cplusplus
}
#endif
#endif /* DARE_GPU_H_ */
