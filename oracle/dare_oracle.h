/*
 * dare_oracle.h -- CPU restatement of DaRe's finite-volume hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm load it.  The product (dare_b200, libdare_gpu.so) never links or calls it.
 *
 * Parity status: the reference (hpc-dave/dare) needs Trilinos, MPI, VTK and
 * Boost and cannot be compiled in this image, so this is a line-by-line
 * restatement of the cited reference files.  It is pinned against the
 * known-answer tests of the reference's own test suite (re-expressed as
 * fixtures under tests/golden/): Grid/test/test_Cartesian_Operators.cpp,
 * Equations/test/test_DDT.cpp, test/test_integration_Cartesian_Trilinos.cpp,
 * MatrixSystem/test/test_TrilinosSolver.cpp and
 * test/test_integration_Cartesian_Field.cpp.
 *
 * Conventions (all from the reference):
 *   - cell ordinal, last active dimension fastest:
 *       ordinal = (i*ny + j)*nz + k      (CartesianRepresentation.inl:87-112)
 *   - ghosted ("local") arrays carry num_ghost layers in every ACTIVE
 *     dimension only (CartesianRepresentation.inl:80-83)
 *   - neighbour slots CENTER=0, WEST=1, EAST=2, SOUTH=3, NORTH=4, BOTTOM=5,
 *     TOP=6 (CartesianMesh.h:67-77); WEST/EAST along x (i), SOUTH/NORTH along
 *     y (j), BOTTOM/TOP along z (k).
 */
#ifndef DARE_ORACLE_H_
#define DARE_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { DOR_C = 0, DOR_W = 1, DOR_E = 2, DOR_S = 3, DOR_N = 4, DOR_B = 5, DOR_T = 6 };
enum { DOR_BC_NONE = 0, DOR_BC_DIRICHLET = 1, DOR_BC_NEUMANN = 2 };
enum { DOR_LIM_CDS = 0, DOR_LIM_UPWIND = 1, DOR_LIM_VANALBADA = 2, DOR_LIM_MINMOD = 3, DOR_LIM_VANLEER = 4 };
enum { DOR_PREC_NONE = 0, DOR_PREC_JACOBI = 1 };

typedef struct {
    int dim;           /* 1, 2 or 3 */
    int num_ghost;     /* ghost layers per active dimension (reference default 2) */
    int64_t n[3];      /* internal resolution; 1 for inactive dimensions */
    double size[3];    /* domain length per dimension */
    int periodic[3];
} dor_grid;

typedef struct {
    dor_grid grid;
    double dt;                  /* > 0: include DDT (implicit Euler) */
    int diffusion;              /* 0 none, 1 scalar D, 2 face arrays */
    double D;
    const double* face_D[3];    /* x-faces (nx+1,ny,nz), y-faces (nx,ny+1,nz), z-faces (nx,ny,nz+1) */
    int convection;             /* 0 none, 1 constant velocity, 2 face velocity arrays */
    int limiter;
    double vel[3];
    const double* face_vel[3];  /* same face layout as face_D */
    int bc_type[6];             /* faces W,E,S,N,B,T */
    double bc_value[6];
    int scheme;                 /* time scheme of the Divergence operators: DOR_SCHEME_* */
    int no_fold;                /* 1: leave the boundary faces unfolded (one term of a composed
                                   functor, folded by the caller after the last term) */
} dor_assembly;

/* Time discretisation of the Divergence operators (TimeDiscretizationSchemes.h:29-76):
 * weights w[0..T]; the implicit coefficients are scaled by w[0] and every
 * explicit level t >= 1 adds w[t] * A * (rhs_E - rhs_W) ... of its face
 * stencil (Divergence_Cartesian.inl:186-205). */
enum { DOR_SCHEME_EULER_BACKWARD = 0, DOR_SCHEME_EULER_FORWARD = 1, DOR_SCHEME_CRANK_NICHOLSON = 2,
       DOR_SCHEME_ADAMS_BASHFORTH = 3, DOR_SCHEME_ADAMS_MOULTON = 4 };
/* Number of explicit levels T and the weights w[0..T]; -1 for an unknown scheme. */
int dor_scheme_weights(int scheme, double w[3]);

typedef struct {
    double tol;        /* absolute tolerance on ||r||_2 (stop criterion RNORM) */
    int max_it;
    int precond;       /* DOR_PREC_NONE / DOR_PREC_JACOBI (right) */
    int iters;         /* out */
    int converged;     /* out */
    int status;        /* out: 0 ok/maxit, else breakdown step (3,4,7,14,20,21) */
    double res;        /* out: last convergence check value */
} dor_solve_info;

int dor_version(void);
int dor_num_threads(void);
void dor_set_threads(int n);

void dor_geometry(const dor_grid* g, double dx[3], double* volume, double area[3]);
int64_t dor_num_cells(const dor_grid* g);
int64_t dor_num_cells_ghosted(const dor_grid* g);
int64_t dor_ordinal_internal(const dor_grid* g, int64_t i, int64_t j, int64_t k);
int64_t dor_internal_to_local(const dor_grid* g, int64_t n_internal);
int64_t dor_global_internal_periodic(const dor_grid* g, int64_t i, int64_t j, int64_t k);

double dor_limiter(int kind, double r);
double dor_diffusion_n0d1(double tau, double zeta, int n_modes);

void dor_exchange_halo(const dor_grid* g, double* phi);
void dor_copy_to_old(const dor_grid* g, double* const* levels, int num_levels);
void dor_copy_to_field(const dor_grid* g, const double* x, double* phi);
void dor_field_to_vector(const dor_grid* g, const double* phi, double* x);

int dor_assemble(const dor_assembly* a, const double* phi_conv, const double* phi_old,
                 double* diag, double* rhs, uint8_t* mask);
int64_t dor_csr_nnz(const dor_grid* g, const uint8_t* mask);
int dor_export_csr(const dor_grid* g, const double* diag, const uint8_t* mask,
                   int64_t* rowptr, int64_t* cols, double* vals);

void dor_spmv(int64_t n, const int64_t* rowptr, const int64_t* cols, const double* vals,
              const double* x, double* y);
double dor_norm2(int64_t n, const double* x);
int dor_bicgstab2(int64_t n, const int64_t* rowptr, const int64_t* cols, const double* vals,
                  const double* b, double* x, dor_solve_info* info);

#ifdef __cplusplus
}
#endif
#endif  /* DARE_ORACLE_H_ */
