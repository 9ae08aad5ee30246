// dare_assembly.cu -- fused per-cell assembly of the implicit step on 1-D
// and 2-D grids, and the launcher of every assembly (3-D grids run the
// staged kernel of dare_assembly3.cu).
//
// One thread per cell evaluates the composed functor of the reference's time
// loops and writes the 7 coefficient diagonals, the rhs and the initial guess:
//     mb  = ddt(field)                 DDT.inl:39-81; Set MatrixBlock_Cartesian.inl:480-497
//     mb += div(TVD(vel) * field)      TVD_Cartesian.inl:185-261; Divergence_Cartesian.inl:139-207
//     mb -= div(D, grad(mb))           Gradient_Cartesian.inl:37-58; Divergence_Cartesian.inl:90-96
//     boundary folding, faces W,E,S,N,B,T (counter_diffusion1D.cpp:123-146):
//         Dirichlet: C -= X; rhs -= 2*bc*X; Remove(X)    Neumann: C += X; Remove(X)
// Every product and sum is evaluated in the reference's order and this file
// is compiled with --fmad=false, so these coefficients are bit-identical to
// the CPU path.
#include "dare_assembly.cuh"

using namespace dare_gpu;

namespace dare_gpu {

__device__ __forceinline__ int64_t face_index(const GridDev& g, int d, int i, int j, int k) {
    switch (d) {
    case 0: return ((int64_t)i * g.n[1] + j) * g.n[2] + k;
    case 1: return ((int64_t)i * (g.n[1] + 1) + j) * g.n[2] + k;
    default: return ((int64_t)i * g.n[1] + j) * (g.n[2] + 1) + k;
    }
}

// ApplyDivergence of a face matrix stencil (Divergence_Cartesian.inl:143-181)
template <int DIM>
__device__ __forceinline__ void apply_divergence(const GridDev& g, const double nb[7], const double cc[7],
                                                 double sc[7]) {
    constexpr int dim = DIM;
    const double* A = g.area;
#pragma unroll
    for (int p = 0; p < 7; p++) sc[p] = 0.;
    sc[DARE_EAST] = A[0] * nb[DARE_EAST];
    sc[DARE_CENTER] = A[0] * cc[DARE_EAST];
    sc[DARE_WEST] = -A[0] * nb[DARE_WEST];
    sc[DARE_CENTER] -= A[0] * cc[DARE_WEST];
    if (dim > 1) {
        sc[DARE_NORTH] = A[1] * nb[DARE_NORTH];
        sc[DARE_CENTER] += A[1] * cc[DARE_NORTH];
        sc[DARE_SOUTH] = -A[1] * nb[DARE_SOUTH];
        sc[DARE_CENTER] -= A[1] * cc[DARE_SOUTH];
    }
    if (dim > 2) {
        sc[DARE_TOP] = A[2] * nb[DARE_TOP];
        sc[DARE_CENTER] += A[2] * cc[DARE_TOP];
        sc[DARE_BOTTOM] = -A[2] * nb[DARE_BOTTOM];
        sc[DARE_CENTER] -= A[2] * cc[DARE_BOTTOM];
    }
}

// One TVD face (TVD_Cartesian.inl:199-258).  The stencil line along the face
// normal is (m2, m1, c0, p1, p2) = phi at offsets -2..+2; `upper` selects the
// upper face.  Writes the face matrix stencil (neighbour, centre, rhs).
__device__ __forceinline__ void tvd_face(bool upper, double m2, double m1, double c0, double p1, double p2,
                                         double v, int limiter, double& nb, double& cf, double& rr) {
    const int vp = v >= 0., vn = !(v >= 0.);
    double pUU, pU, pD;
    if (!upper) {   // UU = i + vn - 2 vp, U = i - vp, D = i - vn
        pUU = vp ? m2 : p1;
        pU = vp ? m1 : c0;
        pD = vp ? c0 : m1;
    } else {        // UU = i + 2 vn - vp, U = i + vn, D = i + vp
        pUU = vp ? m1 : p2;
        pU = vp ? c0 : p1;
        pD = vp ? p1 : c0;
    }
    const double r = (pU - pUU) / (pD - pU);
    const double psi = limiter_value(limiter, r);
    if (!upper) {
        nb = ((double)vp * v) * 1.;
        cf = ((double)vn * v) * 1.;
    } else {
        nb = ((double)vn * v) * 1.;
        cf = ((double)vp * v) * 1.;
    }
    rr = ((-0.5 * psi) * (pD - pU)) * v;
}

// Column-marching assembly: a thread owns one (j,k) column and walks along i
// through `planes` planes, keeping phi(i-2..i+2) and the x-face velocity in
// registers; addresses advance by constant strides (no per-cell index
// division).  The arithmetic per cell is exactly the per-cell functor above.
template <int DIM>
__global__ void __launch_bounds__(256) k_assemble(GridDev g, AsmParams a, const double* __restrict__ phi,
                                                  const double* __restrict__ phi_old, double* __restrict__ diag,
                                                  double* __restrict__ rhs_out, double* __restrict__ x0,
                                                  int planes) {
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y * blockDim.y + threadIdx.y;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    if (jj >= n1 || kk >= n2) return;
    const int i0 = blockIdx.z * planes;
    const int i1 = min(i0 + planes, n0);
    if (i0 >= i1) return;
    const int64_t n = a.dstride;
    const int64_t S0 = (int64_t)g.gn[1] * g.gn[2], S1 = g.gn[2];
    const int64_t nplane = (int64_t)n1 * n2;
    const int64_t jk = (int64_t)jj * n2 + kk;
    int64_t loc = local_index(g, i0, jj, kk);
    int64_t c = (int64_t)i0 * nplane + jk;
    // face-array offsets: x-faces (n0+1, n1, n2), y-faces (n0, n1+1, n2), z-faces (n0, n1, n2+1)
    const int64_t fy_plane = (int64_t)(n1 + 1) * n2, fz_plane = (int64_t)n1 * (n2 + 1);
    int64_t fy_lo = (int64_t)i0 * fy_plane + (int64_t)jj * n2 + kk;
    int64_t fy_up = (int64_t)i0 * fy_plane + (int64_t)upper_face(g, 1, jj) * n2 + kk;
    int64_t fz_lo = (int64_t)i0 * fz_plane + (int64_t)jj * (n2 + 1) + kk;
    int64_t fz_up = (int64_t)i0 * fz_plane + (int64_t)jj * (n2 + 1) + upper_face(g, 2, kk);
    double w0 = phi[loc - 2 * S0], w1 = phi[loc - S0], w2 = phi[loc], w3 = phi[loc + S0], w4 = phi[loc + 2 * S0];
    double vx_lo = 0., Dx_lo = 0.;
    if (a.convection == 2) vx_lo = a.face_vel[0][(int64_t)i0 * nplane + jk];
    if (a.diffusion == 2) Dx_lo = a.face_D[0][(int64_t)i0 * nplane + jk];

    for (int i = i0; i < i1; i++) {
        const int64_t fx_up = (int64_t)upper_face(g, 0, i) * nplane + jk;
        double coef[7];
#pragma unroll
        for (int p = 0; p < 7; p++) coef[p] = a.acc ? diag[p * n + c] : 0.;
        double rhs = a.acc ? rhs_out[c] : 0.;

        if (a.dt > 0.) {                                   // DDT, weights (1, 1)
            const double tt = a.tt;
            if (a.sgn_ddt > 0.) {                           // from zero: C = tt, rhs = 0 + tt phi_old
                coef[DARE_CENTER] += tt;
                rhs += tt * phi_old[loc];
            } else {                                        // MatrixBlock -=: += (-1 s)
                coef[DARE_CENTER] += -1. * tt;
                rhs += -1. * (tt * phi_old[loc]);
            }
        }

        if (a.convection) {                                // TVD * field, then divergence
            double nb[7], cf[7], rr[7];
#pragma unroll
            for (int p = 0; p < 7; p++) nb[p] = cf[p] = rr[p] = 0.;
            double vlo, vup;
            // x (always active)
            if (a.convection == 1) {
                vlo = vup = a.vel[0];
            } else {
                vlo = vx_lo;
                vup = a.face_vel[0][fx_up];
            }
            tvd_face(false, w0, w1, w2, w3, w4, vlo, a.limiter, nb[DARE_WEST], cf[DARE_WEST], rr[DARE_WEST]);
            tvd_face(true, w0, w1, w2, w3, w4, vup, a.limiter, nb[DARE_EAST], cf[DARE_EAST], rr[DARE_EAST]);
            if (DIM > 1) {
                const double m2 = phi[loc - 2 * S1], m1 = phi[loc - S1], p1 = phi[loc + S1], p2 = phi[loc + 2 * S1];
                if (a.convection == 1) {
                    vlo = vup = a.vel[1];
                } else {
                    vlo = a.face_vel[1][fy_lo];
                    vup = a.face_vel[1][fy_up];
                }
                tvd_face(false, m2, m1, w2, p1, p2, vlo, a.limiter, nb[DARE_SOUTH], cf[DARE_SOUTH], rr[DARE_SOUTH]);
                tvd_face(true, m2, m1, w2, p1, p2, vup, a.limiter, nb[DARE_NORTH], cf[DARE_NORTH], rr[DARE_NORTH]);
            }
            if (DIM > 2) {
                const double m2 = phi[loc - 2], m1 = phi[loc - 1], p1 = phi[loc + 1], p2 = phi[loc + 2];
                if (a.convection == 1) {
                    vlo = vup = a.vel[2];
                } else {
                    vlo = a.face_vel[2][fz_lo];
                    vup = a.face_vel[2][fz_up];
                }
                tvd_face(false, m2, m1, w2, p1, p2, vlo, a.limiter, nb[DARE_BOTTOM], cf[DARE_BOTTOM], rr[DARE_BOTTOM]);
                tvd_face(true, m2, m1, w2, p1, p2, vup, a.limiter, nb[DARE_TOP], cf[DARE_TOP], rr[DARE_TOP]);
            }
            double sc[7];
            apply_divergence<DIM>(g, nb, cf, sc);
#pragma unroll
            for (int p = 0; p < 7; p++) sc[p] *= a.w[0];           // s_c *= weight[0]
            double srhs = g.area[0] * (rr[DARE_EAST] - rr[DARE_WEST]);
            if (DIM > 1) srhs += g.area[1] * (rr[DARE_NORTH] - rr[DARE_SOUTH]);
            if (DIM > 2) srhs += g.area[2] * (rr[DARE_TOP] - rr[DARE_BOTTOM]);
            for (int t = 1; t <= a.nexp; t++) {                // explicit levels (copies of level 0)
                srhs += a.w[t] * g.area[0] * (rr[DARE_EAST] - rr[DARE_WEST]);
                if (DIM > 1) srhs += a.w[t] * g.area[1] * (rr[DARE_NORTH] - rr[DARE_SOUTH]);
                if (DIM > 2) srhs += a.w[t] * g.area[2] * (rr[DARE_TOP] - rr[DARE_BOTTOM]);
            }
            if (a.sgn_conv > 0.) {                           // MatrixBlock::Add
#pragma unroll
                for (int p = 0; p < 7; p++) coef[p] += sc[p];
                rhs += srhs;
            } else {                                        // MatrixBlock -=
#pragma unroll
                for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
                rhs += -1. * srhs;
            }
        }

        if (a.diffusion) {                                 // mb -= div(D, grad(mb))
            double Dlo[3], Dup[3];
            if (a.diffusion == 1) {
#pragma unroll
                for (int d = 0; d < 3; d++) Dlo[d] = Dup[d] = a.D;
            } else {
                Dlo[0] = Dx_lo;
                Dup[0] = a.face_D[0][fx_up];
                Dlo[1] = DIM > 1 ? a.face_D[1][fy_lo] : 0.;
                Dup[1] = DIM > 1 ? a.face_D[1][fy_up] : 0.;
                Dlo[2] = DIM > 2 ? a.face_D[2][fz_lo] : 0.;
                Dup[2] = DIM > 2 ? a.face_D[2][fz_up] : 0.;
            }
            double nb[7], cf[7];
#pragma unroll
            for (int p = 0; p < 7; p++) nb[p] = cf[p] = 0.;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                const double dn = a.dn[d];
                const int lo = 2 * d + 1, up = 2 * d + 2;
                nb[lo] = (-dn) * Dlo[d];
                cf[lo] = dn * Dlo[d];
                nb[up] = dn * Dup[d];
                cf[up] = (-dn) * Dup[d];
            }
            double sc[7];
            apply_divergence<DIM>(g, nb, cf, sc);
#pragma unroll
            for (int p = 0; p < 7; p++) sc[p] *= a.w[0];           // s_c *= weight[0]
            if (a.sgn_diff < 0.) {                           // mb -= div(D grad(mb))
#pragma unroll
                for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
                rhs += -1. * 0.;
            } else {
#pragma unroll
                for (int p = 0; p < 7; p++) coef[p] += sc[p];
            }
        }

        const int idx[3] = {i, jj, kk};
#pragma unroll
        for (int d = 0; d < DIM; d++) {                    // boundary folding
            if (g.periodic[d] || !a.fold) continue;
#pragma unroll
            for (int side = 0; side < 2; side++) {
                const int face = 2 * d + 1 + side;
                const bool on_boundary = side == 0 ? (idx[d] == 0) : (idx[d] == g.n[d] - 1);
                if (!on_boundary || (d == 0 && ((a.xint >> side) & 1))) continue;
                const double X = coef[face];
                if (a.bc_type[face - 1] == DARE_BC_DIRICHLET) {
                    coef[DARE_CENTER] -= X;
                    rhs -= 2. * a.bc_value[face - 1] * X;
                } else {
                    coef[DARE_CENTER] += X;
                }
                coef[face] = 0.;
            }
        }
#pragma unroll
        for (int p = 0; p < 7; p++) diag[p * n + c] = coef[p];
        rhs_out[c] = rhs;
        x0[c] = w2;

        // advance one plane
        if (i + 1 < i1) {
            w0 = w1;
            w1 = w2;
            w2 = w3;
            w3 = w4;
            w4 = phi[loc + 3 * S0];
            if (a.convection == 2) vx_lo = a.face_vel[0][fx_up];
            if (a.diffusion == 2) Dx_lo = a.face_D[0][fx_up];
        }
        loc += S0;
        c += nplane;
        fy_lo += fy_plane;
        fy_up += fy_plane;
        fz_lo += fz_plane;
        fz_up += fz_plane;
    }
}

// The conditions on the boundary faces of component c
static void component_bc(const dare_system* s, int c, AsmParams& a) {
    const bool own = !s->bc_type_c.empty();
    for (int f = 0; f < 6; f++) {
        a.bc_type[f] = own ? s->bc_type_c[(size_t)c * 6 + f] : s->bc_type[f];
        a.bc_value[f] = own ? s->bc_value_c[(size_t)c * 6 + f] : s->bc_value[f];
    }
}

// Launch the assembly kernel of the grid's dimension for field component c
// (its field values, its rows).
static int launch_component(dare_system* s, const AsmParams& a, int c, const double* phi, const double* phi_old) {
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->grid->dev;
    const double* pc = phi + (size_t)c * g.ncell_ghosted;
    const double* po = phi_old + (size_t)c * g.ncell_ghosted;
    double* dc = s->diag + (size_t)c * g.ncell;
    double* rc = s->rhs + (size_t)c * g.ncell;
    double* xc = s->x + (size_t)c * g.ncell;
    if (g.dim == 3) return launch_assemble3(ctx, g, a, pc, po, dc, rc, xc);
    // (j,k) tiles of tk x tj columns, runs of `planes` i-planes per block
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int tk = n2 > 16 ? 32 : n2 > 8 ? 16 : n2 > 4 ? 8 : n2 > 2 ? 4 : 1;
    int tj = 256 / tk;
    while (tj > 1 && tj / 2 >= n1) tj /= 2;
    const int gx = (n2 + tk - 1) / tk, gy = (n1 + tj - 1) / tj;
    const int64_t tiles = (int64_t)gx * gy;
    int64_t nchunk = (2 * 8 * (int64_t)ctx->num_sms + tiles - 1) / tiles;
    if (nchunk > n0) nchunk = n0;
    if (nchunk < 1) nchunk = 1;
    int planes = (int)((n0 + nchunk - 1) / nchunk);
    if (planes < 2 && n0 >= 2) planes = 2;
    nchunk = (n0 + planes - 1) / planes;
    const dim3 grid(gx, gy, (unsigned)nchunk), block(tk, tj, 1);
    if (g.dim == 2)
        k_assemble<2><<<grid, block, 0, ctx->stream>>>(g, a, pc, po, dc, rc, xc, planes);
    else
        k_assemble<1><<<grid, block, 0, ctx->stream>>>(g, a, pc, po, dc, rc, xc, planes);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// A COEFFS term: the caller's per-cell values of the 7 slots and the rhs
// (null: 0), set (acc = 0) or added with the term's sign to component c's
// rows.
struct CoefTerm {
    const double* coef[7];
    const double* rhs;
};
__global__ void k_term_coeffs(int64_t n, int64_t dstride, CoefTerm t, double sgn, int acc, double* __restrict__ diag,
                              double* __restrict__ rhs) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 7; q++) {
            const double v = t.coef[q] ? t.coef[q][c] : 0.;
            const double sv = sgn > 0. ? v : -1. * v;
            diag[q * dstride + c] = acc ? diag[q * dstride + c] + sv : sv;
        }
        const double v = t.rhs ? t.rhs[c] : 0.;
        const double sv = sgn > 0. ? v : -1. * v;
        rhs[c] = acc ? rhs[c] + sv : sv;
    }
}

// Geometry, scheme weights and checks shared by both entry points.
static int base_params(dare_system* s, AsmParams& a, const char* who) {
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->grid->dev;
    a.tt = a.dt > 0. ? (g.volume * 1.) / a.dt : 0.;
    a.dstride = s->sdev.ncell;
    a.xint = s->xint;
    a.nexp = scheme_weights(a.scheme, a.w);
    if (a.nexp < 0) return set_error(ctx, DARE_ERR_BAD_ARG, std::string(who) + ": unknown time scheme");
    for (int d = 0; d < 3; d++) a.dn[d] = 1. / g.dx[d];
    for (int d = 0; d < g.dim; d++) {
        if (a.diffusion == 2 && !a.face_D[d]) return set_error(ctx, DARE_ERR_BAD_ARG, std::string(who) + ": face_D missing");
        if (a.convection == 2 && !a.face_vel[d])
            return set_error(ctx, DARE_ERR_BAD_ARG, std::string(who) + ": face_vel missing");
    }
    if (a.diffusion < 0 || a.diffusion > 2 || a.convection < 0 || a.convection > 2 || a.limiter < 0 ||
        a.limiter > DARE_LIMITER_VANLEER || !(a.dt >= 0.))
        return set_error(ctx, DARE_ERR_BAD_ARG, std::string(who) + ": bad descriptor");
    return DARE_OK;
}

static void fused_params(const dare_assembly_desc* desc, AsmParams& a) {
    a.dt = desc->dt;
    a.diffusion = desc->diffusion;
    a.D = desc->D;
    a.convection = desc->convection;
    a.limiter = desc->limiter;
    for (int d = 0; d < 3; d++) {
        a.face_D[d] = desc->face_D[d];
        a.face_vel[d] = desc->face_vel[d];
        a.vel[d] = desc->vel[d];
    }
    a.scheme = desc->scheme;
    // the fused functor: mb = ddt; mb += div(TVD * field); mb -= div(D grad); fold
    a.sgn_ddt = 1.;
    a.sgn_conv = 1.;
    a.sgn_diff = -1.;
    a.acc = 0;
    a.fold = 1;
}

int launch_assemble(dare_system* s, const dare_assembly_desc* desc, const double* phi, const double* phi_old) {
    AsmParams a{};
    fused_params(desc, a);
    int rc = base_params(s, a, "dare_assemble");
    if (rc) return rc;
    for (int c = 0; c < s->ncomp; c++) {
        component_bc(s, c, a);
        if ((rc = launch_component(s, a, c, phi, phi_old))) return rc;
    }
    return DARE_OK;
}

// The fused functor on the planes ib .. ie - 1 of a single-component 3-D
// grid: each plane's coefficients are those of the whole-grid launch, bit for
// bit.  DARE_ERR_UNSUPPORTED on other grids.
int launch_assemble_planes(dare_system* s, const dare_assembly_desc* desc, const double* phi, const double* phi_old,
                           int ib, int ie) {
    const GridDev& g = s->grid->dev;
    if (g.dim != 3 || s->ncomp != 1) return DARE_ERR_UNSUPPORTED;
    AsmParams a{};
    fused_params(desc, a);
    int rc = base_params(s, a, "dare_assemble");
    if (rc) return rc;
    component_bc(s, 0, a);
    return launch_assemble3(s->grid->ctx, g, a, phi, phi_old, s->diag, s->rhs, s->x, ib, ie);
}

// A composed functor (dare_assemble_terms): per component, its terms in
// order -- each one launch that sets or adds its coefficients -- then one
// pass that folds the boundary faces.
static int launch_terms(dare_system* s, const dare_term* terms, int nterms, const double* phi, const double* phi_old) {
    dare_ctx* ctx = s->grid->ctx;
    for (int t = 0; t < nterms; t++) {
        const dare_term& T = terms[t];
        if (T.kind < DARE_TERM_DDT || T.kind > DARE_TERM_COEFFS || T.op < DARE_OP_SET || T.op > DARE_OP_SUB ||
            T.component < -1 || T.component >= s->ncomp)
            return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble_terms: bad term");
        if (T.kind == DARE_TERM_DDT && !(T.dt > 0.))
            return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble_terms: DDT needs dt > 0");
    }
    int rc;
    for (int c = 0; c < s->ncomp; c++) {
        bool started = false;
        for (int t = 0; t < nterms; t++) {
            const dare_term& T = terms[t];
            if (T.component >= 0 && T.component != c) continue;
            if (T.kind == DARE_TERM_COEFFS) {
                CoefTerm ct{};
                for (int q = 0; q < 7; q++) ct.coef[q] = T.coef[q];
                ct.rhs = T.coef_rhs;
                const GridDev& gd = s->grid->dev;
                k_term_coeffs<<<grid_blocks(ctx, gd.ncell, 256, 8), 256, 0, ctx->stream>>>(
                    gd.ncell, s->sdev.ncell, ct, T.op == DARE_OP_SUB ? -1. : 1., started && T.op != DARE_OP_SET,
                    s->diag + (size_t)c * gd.ncell, s->rhs + (size_t)c * gd.ncell);
                DARE_LAUNCHED(ctx);
                started = true;
                continue;
            }
            AsmParams a{};
            a.scheme = T.scheme;
            a.limiter = T.limiter;
            const double sgn = T.op == DARE_OP_SUB ? -1. : 1.;
            a.sgn_ddt = a.sgn_conv = a.sgn_diff = sgn;
            if (T.kind == DARE_TERM_DDT) a.dt = T.dt;
            if (T.kind == DARE_TERM_DIFFUSION) {
                const bool faces = T.face_D[0] || T.face_D[1] || T.face_D[2];
                a.diffusion = faces ? 2 : 1;
                a.D = T.D;
                for (int d = 0; d < 3; d++) a.face_D[d] = T.face_D[d];
            }
            if (T.kind == DARE_TERM_CONVECTION) {
                const bool faces = T.face_vel[0] || T.face_vel[1] || T.face_vel[2];
                a.convection = faces ? 2 : 1;
                for (int d = 0; d < 3; d++) {
                    a.vel[d] = T.vel[d];
                    a.face_vel[d] = T.face_vel[d];
                }
            }
            a.acc = started && T.op != DARE_OP_SET;   // Set starts the component's block afresh
            a.fold = 0;
            if ((rc = base_params(s, a, "dare_assemble_terms"))) return rc;
            component_bc(s, c, a);
            if ((rc = launch_component(s, a, c, phi, phi_old))) return rc;
            started = true;
        }
        // the fold pass (it also zeroes a component that no term touched)
        AsmParams a{};
        a.sgn_ddt = a.sgn_conv = 1.;
        a.sgn_diff = -1.;
        a.acc = started;
        a.fold = 1;
        a.limiter = DARE_LIMITER_CDS;
        if ((rc = base_params(s, a, "dare_assemble_terms"))) return rc;
        component_bc(s, c, a);
        if ((rc = launch_component(s, a, c, phi, phi_old))) return rc;
    }
    return DARE_OK;
}

}  // namespace dare_gpu

extern "C" int dare_assemble(dare_system* s, const dare_assembly_desc* desc, dare_field* field) {
    if (!s || !desc || !field || field->grid != s->grid || field->ncomp != s->ncomp) return DARE_ERR_BAD_ARG;
    cudaSetDevice(s->grid->ctx->device);
    const double* phi = field->level[0];
    const double* phi_old = field->num_levels > 1 ? field->level[1] : field->level[0];
    return dare_gpu::launch_assemble(s, desc, phi, phi_old);
}

extern "C" int dare_assemble_terms(dare_system* s, const dare_term* terms, int nterms, dare_field* field) {
    if (!s || (!terms && nterms > 0) || nterms < 0 || !field || field->grid != s->grid || field->ncomp != s->ncomp)
        return DARE_ERR_BAD_ARG;
    cudaSetDevice(s->grid->ctx->device);
    const double* phi = field->level[0];
    const double* phi_old = field->num_levels > 1 ? field->level[1] : field->level[0];
    return dare_gpu::launch_terms(s, terms, nterms, phi, phi_old);
}
