// dare_assembly.cu -- fused per-cell assembly of the implicit step.
//
// One thread per cell evaluates the composed functor of the reference's time
// loops and writes the 7 coefficient diagonals, the rhs and the initial guess:
//     mb  = ddt(field)                 DDT.inl:39-81; Set MatrixBlock_Cartesian.inl:480-497
//     mb += div(TVD(vel) * field)      TVD_Cartesian.inl:185-261; Divergence_Cartesian.inl:139-207
//     mb -= div(D, grad(mb))           Gradient_Cartesian.inl:37-58; Divergence_Cartesian.inl:90-96
//     boundary folding, faces W,E,S,N,B,T (counter_diffusion1D.cpp:123-146):
//         Dirichlet: C -= X; rhs -= 2*bc*X; Remove(X)    Neumann: C += X; Remove(X)
// Every product and sum is evaluated in the reference's order and this file
// is compiled with --fmad=false, so the coefficients are bit-identical to the
// CPU path.  Algorithmic traffic per cell: phi (8 B, neighbours from cache),
// phi_old (8 B), face velocities (24 B) or face D (24 B) when used, and 72 B
// written (7 diagonals + rhs... + x0).
#include "dare_internal.cuh"

using namespace dare_gpu;

namespace dare_gpu {

struct AsmParams {
    double dt;
    int diffusion;
    double D;
    const double* face_D[3];
    int convection;
    int limiter;
    double vel[3];
    const double* face_vel[3];
    int bc_type[6];
    double bc_value[6];
};

__device__ __forceinline__ double limiter_value(int kind, double r) {
    switch (kind) {
    case DARE_LIMITER_CDS:
        return 1.;
    case DARE_LIMITER_UPWIND:
        return 0.;
    case DARE_LIMITER_VANALBADA: {       // FluxLimiter.h:125-131
        r = isnan(r) ? 0. : r;
        const double r_sqr = r * r;
        return (r + r_sqr) / (1. + r_sqr);
    }
    case DARE_LIMITER_MINMOD: {          // FluxLimiter.h:165-170
        r = isnan(r) ? 0. : r;
        const double m = (1. < r) ? 1. : r;
        return (0. < m) ? m : 0.;
    }
    default: {                            // van Leer: (r+|r|)/(1+|r|), NaN->0, +inf->2, -inf->0
        if (isnan(r)) return 0.;
        if (isinf(r)) return r > 0. ? 2. : 0.;
        const double a = fabs(r);
        return (r + a) / (1. + a);
    }
    }
}

__device__ __forceinline__ int64_t face_index(const GridDev& g, int d, int i, int j, int k) {
    switch (d) {
    case 0: return ((int64_t)i * g.n[1] + j) * g.n[2] + k;
    case 1: return ((int64_t)i * (g.n[1] + 1) + j) * g.n[2] + k;
    default: return ((int64_t)i * g.n[1] + j) * (g.n[2] + 1) + k;
    }
}

__device__ __forceinline__ int upper_face(const GridDev& g, int d, int i) {
    return (g.periodic[d] && i + 1 == g.n[d]) ? 0 : i + 1;
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

template <int DIM>
__global__ void __launch_bounds__(256) k_assemble(GridDev g, AsmParams a, const double* __restrict__ phi,
                                                  const double* __restrict__ phi_old, double* __restrict__ diag,
                                                  double* __restrict__ rhs_out, double* __restrict__ x0) {
    const int64_t n = g.ncell;
    const int64_t lstride[3] = {(int64_t)g.gn[1] * g.gn[2], g.gn[2], 1};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const unsigned cc_ = (unsigned)c, nz = (unsigned)g.n[2], ny = (unsigned)g.n[1];
        const unsigned row = cc_ / nz;
        const int k = (int)(cc_ - row * nz);
        const int i = (int)(row / ny);
        const int j = (int)(row - (unsigned)i * ny);
        const int idx[3] = {i, j, k};
        const int64_t loc = local_index(g, i, j, k);
        double coef[7];
#pragma unroll
        for (int p = 0; p < 7; p++) coef[p] = 0.;
        double rhs = 0.;
        const double phi_c = phi[loc];

        if (a.dt > 0.) {                                   // DDT, weights (1, 1)
            const double tt = (g.volume * 1.) / a.dt;
            coef[DARE_CENTER] = tt;
            rhs = 0. + tt * phi_old[loc];
        }

        if (a.convection) {                                // TVD * field, then divergence
            double nb[7], cf[7], rr[7];
#pragma unroll
            for (int p = 0; p < 7; p++) nb[p] = cf[p] = rr[p] = 0.;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                const int lo = 2 * d + 1, up = 2 * d + 2;
                double vlo, vup;
                if (a.convection == 1) {
                    vlo = vup = a.vel[d];
                } else {
                    int fi[3] = {i, j, k};
                    vlo = a.face_vel[d][face_index(g, d, fi[0], fi[1], fi[2])];
                    fi[d] = upper_face(g, d, fi[d]);
                    vup = a.face_vel[d][face_index(g, d, fi[0], fi[1], fi[2])];
                }
                const int64_t s = lstride[d];
                {   // lower face (TVD_Cartesian.inl:199-227)
                    const int vp = vlo >= 0., vn = !(vlo >= 0.);
                    const double pUU = phi[loc + (int64_t)(vn - 2 * vp) * s];
                    const double pU = phi[loc - (int64_t)vp * s];
                    const double pD = phi[loc - (int64_t)vn * s];
                    const double r = (pU - pUU) / (pD - pU);
                    const double psi = limiter_value(a.limiter, r);
                    nb[lo] = ((double)vp * vlo) * 1.;
                    cf[lo] = ((double)vn * vlo) * 1.;
                    rr[lo] = ((-0.5 * psi) * (pD - pU)) * vlo;
                }
                {   // upper face (TVD_Cartesian.inl:229-258)
                    const int vp = vup >= 0., vn = !(vup >= 0.);
                    const double pUU = phi[loc + (int64_t)(2 * vn - vp) * s];
                    const double pU = phi[loc + (int64_t)vn * s];
                    const double pD = phi[loc + (int64_t)vp * s];
                    const double r = (pU - pUU) / (pD - pU);
                    const double psi = limiter_value(a.limiter, r);
                    nb[up] = ((double)vn * vup) * 1.;
                    cf[up] = ((double)vp * vup) * 1.;
                    rr[up] = ((-0.5 * psi) * (pD - pU)) * vup;
                }
            }
            double sc[7];
            apply_divergence<DIM>(g, nb, cf, sc);
#pragma unroll
            for (int p = 0; p < 7; p++) sc[p] *= 1.;
            double srhs = g.area[0] * (rr[DARE_EAST] - rr[DARE_WEST]);
            if (DIM > 1) srhs += g.area[1] * (rr[DARE_NORTH] - rr[DARE_SOUTH]);
            if (DIM > 2) srhs += g.area[2] * (rr[DARE_TOP] - rr[DARE_BOTTOM]);
#pragma unroll
            for (int p = 0; p < 7; p++) coef[p] += sc[p];       // MatrixBlock::Add
            rhs += srhs;
        }

        if (a.diffusion) {                                 // mb -= div(D, grad(mb))
            double nb[7], cf[7];
#pragma unroll
            for (int p = 0; p < 7; p++) nb[p] = cf[p] = 0.;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                const double dn = 1. / g.dx[d];
                const int lo = 2 * d + 1, up = 2 * d + 2;
                double Dlo, Dup;
                if (a.diffusion == 1) {
                    Dlo = Dup = a.D;
                } else {
                    int fi[3] = {i, j, k};
                    Dlo = a.face_D[d][face_index(g, d, fi[0], fi[1], fi[2])];
                    fi[d] = upper_face(g, d, fi[d]);
                    Dup = a.face_D[d][face_index(g, d, fi[0], fi[1], fi[2])];
                }
                nb[lo] = (-dn) * Dlo;
                cf[lo] = dn * Dlo;
                nb[up] = dn * Dup;
                cf[up] = (-dn) * Dup;
            }
            double sc[7];
            apply_divergence<DIM>(g, nb, cf, sc);
#pragma unroll
            for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
            rhs += -1. * 0.;
        }

#pragma unroll
        for (int d = 0; d < DIM; d++) {                    // boundary folding
            if (g.periodic[d]) continue;
#pragma unroll
            for (int side = 0; side < 2; side++) {
                const int face = 2 * d + 1 + side;
                const bool on_boundary = side == 0 ? (idx[d] == 0) : (idx[d] == g.n[d] - 1);
                if (!on_boundary) continue;
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
        x0[c] = phi_c;
    }
}

int launch_assemble(dare_system* s, const dare_assembly_desc* desc, const double* phi, const double* phi_old) {
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->grid->dev;
    AsmParams a{};
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
    for (int f = 0; f < 6; f++) {
        a.bc_type[f] = s->bc_type[f];
        a.bc_value[f] = s->bc_value[f];
    }
    for (int d = 0; d < g.dim; d++) {
        if (a.diffusion == 2 && !a.face_D[d]) return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: face_D missing");
        if (a.convection == 2 && !a.face_vel[d])
            return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: face_vel missing");
    }
    if (a.diffusion < 0 || a.diffusion > 2 || a.convection < 0 || a.convection > 2 || a.limiter < 0 ||
        a.limiter > DARE_LIMITER_VANLEER)
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: bad descriptor");
    const int blocks = grid_blocks(ctx, g.ncell, 256, 8);
    if (g.dim == 3)
        k_assemble<3><<<blocks, 256, 0, ctx->stream>>>(g, a, phi, phi_old, s->diag, s->rhs, s->x);
    else if (g.dim == 2)
        k_assemble<2><<<blocks, 256, 0, ctx->stream>>>(g, a, phi, phi_old, s->diag, s->rhs, s->x);
    else
        k_assemble<1><<<blocks, 256, 0, ctx->stream>>>(g, a, phi, phi_old, s->diag, s->rhs, s->x);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

}  // namespace dare_gpu

extern "C" int dare_assemble(dare_system* s, const dare_assembly_desc* desc, dare_field* field) {
    if (!s || !desc || !field || field->grid != s->grid) return DARE_ERR_BAD_ARG;
    cudaSetDevice(s->grid->ctx->device);
    const double* phi = field->level[0];
    const double* phi_old = field->num_levels > 1 ? field->level[1] : field->level[0];
    return dare_gpu::launch_assemble(s, desc, phi, phi_old);
}
