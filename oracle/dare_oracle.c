/*
 * dare_oracle.c -- CPU restatement of DaRe's finite-volume hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never part of it.
 * Each function cites the reference file:line whose behaviour it restates
 * (paths relative to the hpc-dave/dare source tree).  The reference itself
 * cannot be built here (Trilinos/MPI/VTK/Boost are absent), so parity is
 * pinned through the reference's own known-answer tests, re-expressed under
 * tests/golden/.
 *
 * Floating-point order of operations follows the reference's stencil algebra
 * term by term so that assembled coefficients are reproducible bit for bit.
 * Compile without -ffast-math and without FMA contraction (see Makefile).
 */
#include "dare_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int dor_version(void) { return 1; }

int dor_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void dor_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Geometry and numbering                                                   */
/* ------------------------------------------------------------------------ */

/* Cartesian<Dim> constructor: CartesianMesh.inl:75-83.
 * cell_width = L/n; cell_volume = 1 * dx * dy * dz (in that order);
 * face_area[d] = cell_volume / cell_width[d]. */
void dor_geometry(const dor_grid* g, double dx[3], double* volume, double area[3]) {
    double v = 1.;
    for (int d = 0; d < 3; d++) {
        dx[d] = 1.;
        area[d] = 0.;
    }
    for (int d = 0; d < g->dim; d++) dx[d] = g->size[d] / (double)g->n[d];
    for (int d = 0; d < g->dim; d++) v *= dx[d];
    for (int d = 0; d < g->dim; d++) area[d] = v / dx[d];
    *volume = v;
}

static void ghosted_dims(const dor_grid* g, int64_t gn[3], int64_t og[3]) {
    for (int d = 0; d < 3; d++) {
        int active = d < g->dim;
        og[d] = active ? g->num_ghost : 0;
        gn[d] = g->n[d] + 2 * og[d];
    }
}

int64_t dor_num_cells(const dor_grid* g) { return g->n[0] * g->n[1] * g->n[2]; }

int64_t dor_num_cells_ghosted(const dor_grid* g) {
    int64_t gn[3], og[3];
    ghosted_dims(g, gn, og);
    return gn[0] * gn[1] * gn[2];
}

/* MapIndexToOrdinalLocalInternal: CartesianRepresentation.inl:371-384
 * (hierarchic sums, last dimension fastest). */
int64_t dor_ordinal_internal(const dor_grid* g, int64_t i, int64_t j, int64_t k) {
    return (i * g->n[1] + j) * g->n[2] + k;
}

/* MapInternalToLocal(LO): CartesianRepresentation.inl:314-331 -- split the
 * internal ordinal into indices, add num_ghost in every dimension, re-number
 * on the ghosted grid. */
int64_t dor_internal_to_local(const dor_grid* g, int64_t n_internal) {
    int64_t gn[3], og[3];
    ghosted_dims(g, gn, og);
    int64_t i = n_internal / (g->n[1] * g->n[2]);
    int64_t rem = n_internal - i * g->n[1] * g->n[2];
    int64_t j = rem / g->n[2];
    int64_t k = rem - j * g->n[2];
    return ((i + og[0]) * gn[1] + (j + og[1])) * gn[2] + (k + og[2]);
}

/* MapIndexToOrdinalGlobalInternal(ind, map_periodic=true):
 * CartesianRepresentation.inl:416-450.  Note the reference wraps every
 * dimension as soon as the grid is periodic in ANY dimension (IsPeriodic(),
 * CartesianMesh.inl:272-277). */
int64_t dor_global_internal_periodic(const dor_grid* g, int64_t i, int64_t j, int64_t k) {
    int64_t ind[3] = {i, j, k};
    int any_periodic = g->periodic[0] || g->periodic[1] || g->periodic[2];
    if (any_periodic) {
        for (int d = 0; d < g->dim; d++) {
            if (ind[d] < 0) ind[d] = g->n[d] + ind[d];
            else if (ind[d] >= g->n[d]) ind[d] = ind[d] - g->n[d];
        }
    }
    return (ind[0] * g->n[1] + ind[1]) * g->n[2] + ind[2];
}

/* ------------------------------------------------------------------------ */
/* Flux limiters: Equations/FluxLimiter.h:41-173, plus van Leer (new)       */
/* ------------------------------------------------------------------------ */

double dor_limiter(int kind, double r) {
    switch (kind) {
    case DOR_LIM_CDS:       /* FluxLimiter.h:62-65 */
        return 1.;
    case DOR_LIM_UPWIND:    /* FluxLimiter.h:92-95 */
        return 0.;
    case DOR_LIM_VANALBADA: { /* FluxLimiter.h:125-131: NaN -> 0 */
        r = isnan(r) ? 0. : r;
        const double r_sqr = r * r;
        return (r + r_sqr) / (1. + r_sqr);
    }
    case DOR_LIM_MINMOD: {  /* FluxLimiter.h:165-170: max(0, min(r, 1)), NaN -> 0 */
        r = isnan(r) ? 0. : r;
        double m = (1. < r) ? 1. : r;          /* std::min(r, ONE) */
        return (0. < m) ? m : 0.;              /* std::max(ZERO, m) */
    }
    case DOR_LIM_VANLEER: { /* not in the reference: psi = (r+|r|)/(1+|r|) */
        if (isnan(r)) return 0.;
        if (isinf(r)) return r > 0. ? 2. : 0.;
        const double a = fabs(r);
        return (r + a) / (1. + a);
    }
    default:
        return 0.;
    }
}

/* AnalyticalSolutions/Diffusion.h:46-58 */
double dor_diffusion_n0d1(double tau, double zeta, int n_modes) {
    double phi_inf = 1.;
    double phi_tr = 0.;
    for (int n = 0; n < n_modes; ++n) {
        double npi = (n + 0.5) * M_PI;
        phi_tr += 2 * cos(n * M_PI) / npi * exp(-npi * npi * tau) * cos(npi * zeta);
    }
    return phi_inf - phi_tr;
}

/* ------------------------------------------------------------------------ */
/* Field plumbing                                                           */
/* ------------------------------------------------------------------------ */

/* Field::ExchangeHaloCells on one rank (Field.inl:100-103 -> HaloBuffer).
 * The halo IDs (CartesianRepresentation.inl:132-204) contain only ghost cells
 * that leave the internal range in exactly ONE dimension (count > 1 ->
 * skipped) and whose periodic image is internal; those receive the value of
 * the periodic image.  Physical-boundary ghosts and edge/corner ghosts are
 * left untouched. */
void dor_exchange_halo(const dor_grid* g, double* phi) {
    int64_t gn[3], og[3];
    ghosted_dims(g, gn, og);
    const int64_t total = gn[0] * gn[1] * gn[2];
#pragma omp parallel for schedule(static)
    for (int64_t o = 0; o < total; o++) {
        int64_t ind[3];
        ind[0] = o / (gn[1] * gn[2]);
        ind[1] = (o / gn[2]) % gn[1];
        ind[2] = o % gn[2];
        int out_count = 0, out_dim = -1;
        for (int d = 0; d < g->dim; d++) {
            if (ind[d] < og[d] || ind[d] >= og[d] + g->n[d]) {
                out_count++;
                out_dim = d;
            }
        }
        if (out_count != 1 || !g->periodic[out_dim]) continue;
        int64_t src[3] = {ind[0], ind[1], ind[2]};
        if (src[out_dim] < og[out_dim]) src[out_dim] += g->n[out_dim];
        else src[out_dim] -= g->n[out_dim];
        phi[o] = phi[(src[0] * gn[1] + src[1]) * gn[2] + src[2]];
    }
}

/* Field::CopyDataVectorsToOldTimeStep: Field.inl:88-93 (level n <- n-1,
 * cascading from the oldest level). */
void dor_copy_to_old(const dor_grid* g, double* const* levels, int num_levels) {
    const int64_t total = dor_num_cells_ghosted(g);
    for (int n = num_levels - 1; n > 0; n--)
        memcpy(levels[n], levels[n - 1], (size_t)total * sizeof(double));
}

/* Trilinos::CopyTo: Trilinos.inl:166-177 (solution -> ghosted field). */
void dor_copy_to_field(const dor_grid* g, const double* x, double* phi) {
    const int64_t n = dor_num_cells(g);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; c++) phi[dor_internal_to_local(g, c)] = x[c];
}

/* Initial guess: BuildNew copies the field value of every internal cell into
 * x (MatrixBlockBase initial guess, Trilinos.inl:318-327). */
void dor_field_to_vector(const dor_grid* g, const double* phi, double* x) {
    const int64_t n = dor_num_cells(g);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; c++) x[c] = phi[dor_internal_to_local(g, c)];
}

/* ------------------------------------------------------------------------ */
/* Assembly                                                                 */
/* ------------------------------------------------------------------------ */

static int64_t face_index(const dor_grid* g, int d, int64_t i, int64_t j, int64_t k) {
    switch (d) {
    case 0: return (i * g->n[1] + j) * g->n[2] + k;
    case 1: return (i * (g->n[1] + 1) + j) * g->n[2] + k;
    default: return (i * g->n[1] + j) * (g->n[2] + 1) + k;
    }
}

/* Upper face of cell index i along d.  On a periodic dimension the staggered
 * field has n faces and its halo wraps (CartesianRepresentation.inl:64-76),
 * so face n is face 0. */
static int64_t upper_face(const dor_grid* g, int d, int64_t i) {
    return (g->periodic[d] && i + 1 == g->n[d]) ? 0 : i + 1;
}

int dor_scheme_weights(int scheme, double w[3]) {
    /* TimeDiscretizationSchemes.h: EULER_BACKWARD :29-36 (1), EULER_FORWARD
     * :38-45 (0, 1), CRANK_NICHOLSON :47-54 (0.5, 0.5), ADAMS_BASHFORT :56-65
     * (0, 1.5, -0.5), ADAMS_MOULTON :67-76 (5/12, 8/12, -1/12) */
    w[0] = w[1] = w[2] = 0.;
    switch (scheme) {
    case DOR_SCHEME_EULER_BACKWARD: w[0] = 1.; return 0;
    case DOR_SCHEME_EULER_FORWARD: w[0] = 0.; w[1] = 1.; return 1;
    case DOR_SCHEME_CRANK_NICHOLSON: w[0] = 0.5; w[1] = 0.5; return 1;
    case DOR_SCHEME_ADAMS_BASHFORTH: w[0] = 0.; w[1] = 1.5; w[2] = -0.5; return 2;
    case DOR_SCHEME_ADAMS_MOULTON: w[0] = 5. / 12.; w[1] = 8. / 12.; w[2] = -1. / 12.; return 2;
    default: return -1;
    }
}

/* One cell of the composed user functor
 *     mb  = ddt(field);                      DDT.inl:39-81, Set  MatrixBlock_Cartesian.inl:480-497
 *     mb += div(TVD(vel) * field);           TVD_Cartesian.inl:185-261, Divergence_Cartesian.inl:139-207
 *     mb -= div(D, grad(mb));                Gradient_Cartesian.inl:37-58, Divergence_Cartesian.inl:90-96,
 *                                            MatrixBlock_Cartesian.inl:588-593
 *     boundary folding (W,E,S,N,B,T order):  counter_diffusion1D.cpp:123-146
 *         Dirichlet: C -= X; rhs -= 2*bc*X; Remove(X)
 *         Neumann:   C += X; Remove(X)
 * coef[] holds the 7 slots CENTER..TOP; removed slots are written as 0 and
 * cleared in the mask (bit p = slot p). */
static void assemble_cell(const dor_assembly* a, const double dx[3], double V, const double A[3],
                          const int64_t gn[3], const int64_t og[3],
                          const double* phi_conv, const double* phi_old,
                          int64_t i, int64_t j, int64_t k, double coef[7], double* rhs_out,
                          uint8_t* mask_out) {
    const dor_grid* g = &a->grid;
    const int dim = g->dim;
    const int64_t idx[3] = {i, j, k};
    const int64_t loc = ((i + og[0]) * gn[1] + (j + og[1])) * gn[2] + (k + og[2]);
    const int64_t lstride[3] = {gn[1] * gn[2], gn[2], 1};
    uint8_t mask = 1;
    for (int d = 0; d < dim; d++) mask |= (uint8_t)((1u << (2 * d + 1)) | (1u << (2 * d + 2)));
    double w[3];
    const int T = dor_scheme_weights(a->scheme, w);
    for (int p = 0; p < 7; p++) coef[p] = 0.;
    double rhs = 0.;

    /* DDT with timeschemes::IMPLICIT weights (1,1) (DDT.h:39-48):
     * transient = volume * weights / dt; center = transient[0];
     * rhs = 0 + transient[1] * phi_old(local ordinal). */
    if (a->dt > 0.) {
        const double tt0 = (V * 1.) / a->dt;
        const double tt1 = (V * 1.) / a->dt;
        coef[DOR_C] = tt0;
        rhs = 0. + tt1 * phi_old[loc];
    }

    /* Convection: TVD<Cartesian,SC,Limiter>::operator* then Divergence with
     * the scheme's weights (EULER_BACKWARD: weight 1), then MatrixBlock::Add. */
    if (a->convection) {
        double nb[7], cc[7], rr[7];
        for (int p = 0; p < 7; p++) nb[p] = cc[p] = rr[p] = 0.;
        for (int d = 0; d < dim; d++) {
            const int lo = 2 * d + 1, up = 2 * d + 2;
            double vlo, vup;
            if (a->convection == 1) {
                vlo = vup = a->vel[d];          /* TVD_Cartesian.inl:40-53 */
            } else {                              /* face velocities: TVD_Cartesian.inl:26-38 */
                int64_t fi[3] = {i, j, k};
                vlo = a->face_vel[d][face_index(g, d, fi[0], fi[1], fi[2])];
                fi[d] = upper_face(g, d, fi[d]);
                vup = a->face_vel[d][face_index(g, d, fi[0], fi[1], fi[2])];
            }
            const int64_t s = lstride[d];
            /* lower face: TVD_Cartesian.inl:199-227 */
            {
                const int vp = vlo >= 0., vn = !(vlo >= 0.);
                const int64_t iUU = loc + (int64_t)(vn - 2 * vp) * s;
                const int64_t iU = loc - (int64_t)vp * s;
                const int64_t iD = loc - (int64_t)vn * s;
                const double pUU = phi_conv[iUU], pU = phi_conv[iU], pD = phi_conv[iD];
                const double r = (pU - pUU) / (pD - pU);
                const double psi = dor_limiter(a->limiter, r);
                nb[lo] = ((double)vp * vlo) * 1.;
                cc[lo] = ((double)vn * vlo) * 1.;
                rr[lo] = ((-0.5 * psi) * (pD - pU)) * vlo;
            }
            /* upper face: TVD_Cartesian.inl:229-258 */
            {
                const int vp = vup >= 0., vn = !(vup >= 0.);
                const int64_t iUU = loc + (int64_t)(2 * vn - vp) * s;
                const int64_t iU = loc + (int64_t)vn * s;
                const int64_t iD = loc + (int64_t)vp * s;
                const double pUU = phi_conv[iUU], pU = phi_conv[iU], pD = phi_conv[iD];
                const double r = (pU - pUU) / (pD - pU);
                const double psi = dor_limiter(a->limiter, r);
                nb[up] = ((double)vn * vup) * 1.;
                cc[up] = ((double)vp * vup) * 1.;
                rr[up] = ((-0.5 * psi) * (pD - pU)) * vup;
            }
        }
        /* ApplyDivergence: Divergence_Cartesian.inl:143-197 */
        double sc[7], srhs;
        for (int p = 0; p < 7; p++) sc[p] = 0.;
        sc[DOR_E] = A[0] * nb[DOR_E];
        sc[DOR_C] = A[0] * cc[DOR_E];
        sc[DOR_W] = -A[0] * nb[DOR_W];
        sc[DOR_C] -= A[0] * cc[DOR_W];
        if (dim > 1) {
            sc[DOR_N] = A[1] * nb[DOR_N];
            sc[DOR_C] += A[1] * cc[DOR_N];
            sc[DOR_S] = -A[1] * nb[DOR_S];
            sc[DOR_C] -= A[1] * cc[DOR_S];
        }
        if (dim > 2) {
            sc[DOR_T] = A[2] * nb[DOR_T];
            sc[DOR_C] += A[2] * cc[DOR_T];
            sc[DOR_B] = -A[2] * nb[DOR_B];
            sc[DOR_C] -= A[2] * cc[DOR_B];
        }
        for (int p = 0; p < 7; p++) sc[p] *= w[0];  /* s_c *= weight[0] */
        srhs = A[0] * (rr[DOR_E] - rr[DOR_W]);
        if (dim > 1) srhs += A[1] * (rr[DOR_N] - rr[DOR_S]);
        if (dim > 2) srhs += A[2] * (rr[DOR_T] - rr[DOR_B]);
        /* explicit levels: copies of the level-0 face stencil (f[t] = f[0],
         * Divergence_Cartesian.inl:61-62), weighted (:196-205) */
        for (int t = 1; t <= T; t++) {
            srhs += w[t] * A[0] * (rr[DOR_E] - rr[DOR_W]);
            if (dim > 1) srhs += w[t] * A[1] * (rr[DOR_N] - rr[DOR_S]);
            if (dim > 2) srhs += w[t] * A[2] * (rr[DOR_T] - rr[DOR_B]);
        }
        /* MatrixBlock::Add: MatrixBlock_Cartesian.inl:527-546 */
        for (int p = 0; p < 7; p++) coef[p] += sc[p];
        rhs += srhs;
    }

    /* Diffusion: Gradient matrix form (Gradient_Cartesian.inl:37-58) scaled
     * by D (Divergence::Multiply(SC), Divergence_Cartesian.inl:90-96, or a
     * FaceValueStencil, Stencils_Cartesian.inl:709-716), ApplyDivergence,
     * then mb -= s (MatrixBlock_Cartesian.inl:588-593). */
    if (a->diffusion) {
        double nb[7], cc[7];
        for (int p = 0; p < 7; p++) nb[p] = cc[p] = 0.;
        for (int d = 0; d < dim; d++) {
            const double dn = 1. / dx[d];
            const int lo = 2 * d + 1, up = 2 * d + 2;
            double Dlo, Dup;
            if (a->diffusion == 1) {
                Dlo = Dup = a->D;
            } else {
                int64_t fi[3] = {i, j, k};
                Dlo = a->face_D[d][face_index(g, d, fi[0], fi[1], fi[2])];
                fi[d] = upper_face(g, d, fi[d]);
                Dup = a->face_D[d][face_index(g, d, fi[0], fi[1], fi[2])];
            }
            nb[lo] = (-dn) * Dlo;
            cc[lo] = dn * Dlo;
            nb[up] = dn * Dup;
            cc[up] = (-dn) * Dup;
        }
        double sc[7];
        for (int p = 0; p < 7; p++) sc[p] = 0.;
        sc[DOR_E] = A[0] * nb[DOR_E];
        sc[DOR_C] = A[0] * cc[DOR_E];
        sc[DOR_W] = -A[0] * nb[DOR_W];
        sc[DOR_C] -= A[0] * cc[DOR_W];
        if (dim > 1) {
            sc[DOR_N] = A[1] * nb[DOR_N];
            sc[DOR_C] += A[1] * cc[DOR_N];
            sc[DOR_S] = -A[1] * nb[DOR_S];
            sc[DOR_C] -= A[1] * cc[DOR_S];
        }
        if (dim > 2) {
            sc[DOR_T] = A[2] * nb[DOR_T];
            sc[DOR_C] += A[2] * cc[DOR_T];
            sc[DOR_B] = -A[2] * nb[DOR_B];
            sc[DOR_C] -= A[2] * cc[DOR_B];
        }
        for (int p = 0; p < 7; p++) sc[p] *= w[0];  /* s_c *= weight[0] */
        /* the gradient stencil carries no rhs: the diffusion rhs, explicit
         * levels included, is +0 */
        for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
        rhs += -1. * 0.;
    }

    /* Boundary folding on non-periodic faces, order W,E,S,N,B,T. */
    for (int d = 0; d < dim; d++) {
        if (g->periodic[d]) continue;
        for (int side = 0; side < 2; side++) {
            const int face = 2 * d + 1 + side;
            const int on_boundary = side == 0 ? (idx[d] == 0) : (idx[d] == g->n[d] - 1);
            if (!on_boundary) continue;
            mask &= (uint8_t)~(1u << face);
            if (a->no_fold) continue;
            const double X = coef[face];
            if (a->bc_type[face - 1] == DOR_BC_DIRICHLET) {
                coef[DOR_C] -= X;
                rhs -= 2. * a->bc_value[face - 1] * X;
            } else {
                coef[DOR_C] += X;
            }
            coef[face] = 0.;
        }
    }
    *rhs_out = rhs;
    *mask_out = mask;
}

/* Returns 0 on success, -1 on an invalid description (a non-periodic active
 * face without a Dirichlet/Neumann condition, or a resolution <= num_ghost,
 * which the reference rejects in CartesianMesh.inl:60-69). */
int dor_assemble(const dor_assembly* a, const double* phi_conv, const double* phi_old,
                 double* diag, double* rhs, uint8_t* mask) {
    const dor_grid* g = &a->grid;
    double w[3];
    if (dor_scheme_weights(a->scheme, w) < 0) return -1;
    for (int d = 0; d < g->dim; d++) {
        if (g->n[d] <= g->num_ghost) return -1;
        if (!g->periodic[d]) {
            if (a->bc_type[2 * d] == DOR_BC_NONE || a->bc_type[2 * d + 1] == DOR_BC_NONE) return -1;
        }
    }
    double dx[3], V, A[3];
    dor_geometry(g, dx, &V, A);
    int64_t gn[3], og[3];
    ghosted_dims(g, gn, og);
    const int64_t ncell = dor_num_cells(g);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < ncell; c++) {
        const int64_t i = c / (g->n[1] * g->n[2]);
        const int64_t j = (c / g->n[2]) % g->n[1];
        const int64_t k = c % g->n[2];
        double coef[7], r;
        uint8_t m;
        assemble_cell(a, dx, V, A, gn, og, phi_conv, phi_old, i, j, k, coef, &r, &m);
        for (int p = 0; p < 7; p++) diag[(int64_t)p * ncell + c] = coef[p];
        rhs[c] = r;
        if (mask) mask[c] = m;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* CSR export (MatrixBlock::Finalize + Tpetra fillComplete)                 */
/* ------------------------------------------------------------------------ */

int64_t dor_csr_nnz(const dor_grid* g, const uint8_t* mask) {
    const int64_t n = dor_num_cells(g);
    int64_t nnz = 0;
#pragma omp parallel for reduction(+ : nnz) schedule(static)
    for (int64_t c = 0; c < n; c++) nnz += __builtin_popcount(mask[c]);
    return nnz;
}

/* Finalize (MatrixBlock_Cartesian.inl:127-240) emits W,S,B,C,T,N,E with
 * global periodic columns; Tpetra's fillComplete sorts each row by column
 * (the order PrintRow shows, Trilinos.inl:185-212). rowptr has n+1 entries. */
int dor_export_csr(const dor_grid* g, const double* diag, const uint8_t* mask,
                   int64_t* rowptr, int64_t* cols, double* vals) {
    const int64_t n = dor_num_cells(g);
    rowptr[0] = 0;
    for (int64_t c = 0; c < n; c++) rowptr[c + 1] = rowptr[c] + __builtin_popcount(mask[c]);
    static const int emit_order[7] = {DOR_W, DOR_S, DOR_B, DOR_C, DOR_T, DOR_N, DOR_E};
    static const int off[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0},
                                  {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; c++) {
        const int64_t i = c / (g->n[1] * g->n[2]);
        const int64_t j = (c / g->n[2]) % g->n[1];
        const int64_t k = c % g->n[2];
        int64_t pos = rowptr[c];
        int64_t rc[7];
        double rv[7];
        int cnt = 0;
        for (int e = 0; e < 7; e++) {
            const int p = emit_order[e];
            if (!(mask[c] & (1u << p))) continue;
            rc[cnt] = dor_global_internal_periodic(g, i + off[p][0], j + off[p][1], k + off[p][2]);
            rv[cnt] = diag[(int64_t)p * n + c];
            cnt++;
        }
        /* insertion sort by column */
        for (int a1 = 1; a1 < cnt; a1++) {
            int64_t kc = rc[a1];
            double kv = rv[a1];
            int b1 = a1 - 1;
            while (b1 >= 0 && rc[b1] > kc) {
                rc[b1 + 1] = rc[b1];
                rv[b1 + 1] = rv[b1];
                b1--;
            }
            rc[b1 + 1] = kc;
            rv[b1 + 1] = kv;
        }
        for (int e = 0; e < cnt; e++) {
            cols[pos + e] = rc[e];
            vals[pos + e] = rv[e];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* BiCGStab(2): MatrixSystem/BiCGStab2.inl:166-582                           */
/* ------------------------------------------------------------------------ */

void dor_spmv(int64_t n, const int64_t* rowptr, const int64_t* cols, const double* vals,
              const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; r++) {
        double s = 0.;
        for (int64_t p = rowptr[r]; p < rowptr[r + 1]; p++) s += vals[p] * x[cols[p]];
        y[r] = s;
    }
}

static double dot(int64_t n, const double* a, const double* b) {
    double s = 0.;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

double dor_norm2(int64_t n, const double* x) { return sqrt(dot(n, x, x)); }

/* Tpetra MultiVector::update(alpha, A, beta): this = beta*this + alpha*A */
static void update1(int64_t n, double* y, double alpha, const double* a, double beta) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) y[i] = alpha * a[i] + beta * y[i];
}

/* update(alpha, A, beta, B, gamma): this = gamma*this + alpha*A + beta*B */
static void update2(int64_t n, double* z, double alpha, const double* a, double beta,
                    const double* b, double gamma) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) z[i] = alpha * a[i] + beta * b[i] + gamma * z[i];
}

static void assign(int64_t n, double* y, const double* x) { memcpy(y, x, (size_t)n * sizeof(double)); }

/* Jacobi (Ifpack2 RELAXATION, one sweep, damping 1, zero start): Y = D^-1 X
 * with D^-1 precomputed as 1/diag. */
static void apply_prec(int64_t n, const double* inv_diag, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) y[i] = inv_diag[i] * x[i];
}

int dor_bicgstab2(int64_t n, const int64_t* rowptr, const int64_t* cols, const double* vals,
                  const double* B, double* x, dor_solve_info* info) {
    const double tol = info->tol;
    const int max_iteration = info->max_it;
    const int right = info->precond == DOR_PREC_JACOBI;
    info->status = 0;
    info->converged = 0;
    info->iters = 0;

    double* inv_diag = NULL;
    double* work = (double*)malloc((size_t)n * 13 * sizeof(double));
    if (!work) return -1;
    double *x0 = work, *r = work + n, *r_hat_0 = work + 2 * n, *u = work + 3 * n, *v = work + 4 * n,
           *s = work + 5 * n, *w = work + 6 * n, *t = work + 7 * n, *tmp = work + 8 * n;
    if (right) {
        inv_diag = (double*)malloc((size_t)n * sizeof(double));
        for (int64_t row = 0; row < n; row++) {
            double d = 0.;
            for (int64_t p = rowptr[row]; p < rowptr[row + 1]; p++)
                if (cols[p] == row) d = vals[p];
            inv_diag[row] = 1. / d;
        }
    }

    int k = 0;
    double alpha = 0.;
    double rho[2] = {0., 0.};
    double gamma = 0., beta = 0.;
    long double omega_1 = 0.0L, omega_2 = 0.0L, mu = 0.0L, nu = 0.0L, tau = 0.0L;
    double r_norm_0, convergence_check = 0.;
    const double normalizer = 1.;  /* stop_criteria = RNORM (BiCGStab2.inl:34, 254-257) */
    const double ONE = 1.;

    assign(n, x0, x);
    assign(n, r, B);
    if (right) {  /* BiCGStab2.inl:258-261 */
        apply_prec(n, inv_diag, x0, tmp);
        assign(n, x0, tmp);
    }
    /* (0) r = r_hat_0 = b - A x0 */
    dor_spmv(n, rowptr, cols, vals, x0, v);
    update1(n, r, -ONE, v, ONE);
    assign(n, r_hat_0, r);
    /* (1) */
    memset(u, 0, (size_t)n * sizeof(double));
    memset(v, 0, (size_t)n * sizeof(double));
    memset(w, 0, (size_t)n * sizeof(double));
    rho[0] = omega_1 = omega_2 = ONE;
    alpha = 0.;  /* the reference leaves alpha at its initial 0 (BiCGStab2.inl:182) */

    r_norm_0 = dor_norm2(n, r);
    convergence_check = r_norm_0 / normalizer;
    if (convergence_check < tol) {
        info->iters = k;
        info->res = convergence_check;
        info->converged = 1;
        assign(n, x, x0);
        free(work);
        free(inv_diag);
        return 0;
    }
    ++k;

#define APPLY_OP(src, dst)                                     \
    do {                                                        \
        if (right) {                                            \
            apply_prec(n, inv_diag, src, tmp);                  \
            dor_spmv(n, rowptr, cols, vals, tmp, dst);          \
        } else {                                                \
            dor_spmv(n, rowptr, cols, vals, src, dst);          \
        }                                                       \
    } while (0)

    while (1) {
        if (k > max_iteration) break;
        /* (3) */
        rho[0] = (double)(-omega_2 * (long double)rho[0]);
        if (rho[0] == 0.0) { info->status = 3; break; }
        /* (4) */
        rho[1] = dot(n, r_hat_0, r);
        beta = alpha * rho[1] / rho[0];
        rho[0] = rho[1];
        if (rho[0] == 0.0) { info->status = 4; break; }
        /* (5) */
        update1(n, u, ONE, r, -beta);
        /* (6) */
        APPLY_OP(u, v);
        /* (7) */
        gamma = dot(n, v, r_hat_0);
        if (gamma == 0.0) { info->status = 7; break; }
        alpha = rho[0] / gamma;
        /* (8) */
        update1(n, r, -alpha, v, ONE);
        /* (9) */
        APPLY_OP(r, s);
        /* (10) */
        update1(n, x, alpha, u, 1.);
        /* (11) */
        rho[1] = dot(n, r_hat_0, s);
        beta = alpha * rho[1] / rho[0];
        rho[0] = rho[1];
        /* (12) */
        update1(n, v, ONE, s, -beta);
        /* (13) */
        APPLY_OP(v, w);
        /* (14) */
        gamma = dot(n, w, r_hat_0);
        if (gamma == 0.0) { info->status = 14; break; }
        alpha = rho[0] / gamma;
        /* (15) */
        update1(n, u, 1., r, -beta);
        /* (16) */
        update1(n, r, -alpha, v, ONE);
        /* (17) */
        update1(n, s, -alpha, w, ONE);
        /* (18) */
        APPLY_OP(s, t);
        /* (19), (20) */
        omega_1 = dot(n, r, s);
        mu = dot(n, s, s);
        nu = dot(n, s, t);
        tau = dot(n, t, t);
        omega_2 = dot(n, r, t);
        if (mu == 0.) { info->status = 20; break; }
        /* (21) */
        tau -= nu * nu / mu;
        if (tau == 0.0) {
            /* BiCGStab2.inl:407-424: true residual check, early return */
            if (right) {
                apply_prec(n, inv_diag, x, tmp);
                assign(n, x, tmp);
            }
            assign(n, r, B);
            dor_spmv(n, rowptr, cols, vals, x, v);
            update1(n, r, -1., v, 1.);
            convergence_check = dor_norm2(n, r) / normalizer;
            if (convergence_check <= tol) {
                info->converged = 1;
                info->iters = k;
                info->res = convergence_check;
                free(work);
                free(inv_diag);
                return 0;
            }
            /* not converged: the reference breaks to the common exit, which
             * applies the right preconditioner a second time */
            info->status = 21;
            break;
        }
        /* (22), (23) */
        omega_2 = (omega_2 - (nu * omega_1) / mu) / tau;
        omega_1 = (omega_1 - nu * omega_2) / mu;
        /* (24) */
        update2(n, x, (double)omega_1, r, (double)omega_2, s, ONE);
        update1(n, x, alpha, u, ONE);
        /* (25) */
        update2(n, r, (double)(-omega_1), s, (double)(-omega_2), t, ONE);
        convergence_check = dor_norm2(n, r) / normalizer;
        if (convergence_check <= tol && k > 1) break;
        update2(n, u, (double)(-omega_1), v, (double)(-omega_2), w, ONE);
        ++k;
    }
#undef APPLY_OP
    if (right) {
        apply_prec(n, inv_diag, x, tmp);
        assign(n, x, tmp);
    }
    info->iters = k;
    info->res = convergence_check;
    info->converged = convergence_check <= tol;
    free(work);
    free(inv_diag);
    return 0;
}
