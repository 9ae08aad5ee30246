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
    double tt;      // (V * 1) / dt, the DDT weight (evaluated once on the host: same IEEE result)
    double dn[3];   // 1 / dx per dimension (Gradient_Cartesian.inl:30-34)
    int64_t dstride; // elements between two coefficient slots (cells x field components)
    int scheme;     // DARE_SCHEME_* of the div(...) terms
    int nexp;       // its explicit levels T
    double w[3];    // its weights w[0..T] (TimeDiscretizationSchemes.h:29-76)
};

// Weights of the Divergence time schemes (TimeDiscretizationSchemes.h:29-76);
// returns the number of explicit levels, -1 for an unknown scheme.
static int scheme_weights(int scheme, double w[3]) {
    w[0] = w[1] = w[2] = 0.;
    switch (scheme) {
    case DARE_SCHEME_EULER_BACKWARD: w[0] = 1.; return 0;
    case DARE_SCHEME_EULER_FORWARD: w[1] = 1.; return 1;
    case DARE_SCHEME_CRANK_NICHOLSON: w[0] = 0.5; w[1] = 0.5; return 1;
    case DARE_SCHEME_ADAMS_BASHFORTH: w[1] = 1.5; w[2] = -0.5; return 2;
    case DARE_SCHEME_ADAMS_MOULTON: w[0] = 5. / 12.; w[1] = 8. / 12.; w[2] = -1. / 12.; return 2;
    default: return -1;
    }
}

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
        for (int p = 0; p < 7; p++) coef[p] = 0.;
        double rhs = 0.;

        if (a.dt > 0.) {                                   // DDT, weights (1, 1)
            const double tt = a.tt;
            coef[DARE_CENTER] = tt;
            rhs = 0. + tt * phi_old[loc];
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
#pragma unroll
            for (int p = 0; p < 7; p++) coef[p] += sc[p];       // MatrixBlock::Add
            rhs += srhs;
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
#pragma unroll
            for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
            rhs += -1. * 0.;
        }

        const int idx[3] = {i, jj, kk};
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

// The limited flux correction of one TVD face, rr = -0.5 psi(r) (phi_D -
// phi_U) v (TVD_Cartesian.inl:199-258), from the four values along the face
// normal, lower side first: (a, b, c, d) = phi at f - 3/2, f - 1/2, f + 1/2,
// f + 3/2.  tvd_face(false, a, b, c, d, .) of the upper cell and
// tvd_face(true, ., a, b, c, d) of the lower cell select the same upwind
// values from these, so both cells of a face get the same rr from here.
template <int LIM>
__device__ __forceinline__ double face_rr(double a, double b, double c, double d, double v) {
    const int vp = v >= 0.;
    const double pUU = vp ? a : d, pU = vp ? b : c, pD = vp ? c : b;
    const double r = (pU - pUU) / (pD - pU);
    const double psi = limiter_value(LIM, r);
    return ((-0.5 * psi) * (pD - pU)) * v;
}

// Face-sharing assembly of 3-D grids.  An interior face's rr (two IEEE
// divisions and the limiter) is the same for its two cells, so a cell
// evaluates only its upper faces E, N, T and takes
//   W  from its own E face one plane earlier (the march along i),
//   S  from the N face of the row below (shared memory),
//   B  from the T face of the lane below (a warp shuffle);
// the first plane of a run evaluates W itself, the first row of a block S.
// A warp covers 31 cells of a k row: lane 0 is the cell below them and only
// supplies its T face.  Every coefficient comes from the same operations on the same operands as
// the per-cell evaluation of k_assemble, so the results are bit-identical.
// The kernel is latency-bound (FP64 divisions, loads): it is held to 64
// registers so four blocks share an SM (a few spilled words; 0.79 ms at 256^3
// against 0.86 ms with 80 registers at three blocks, no gain at five).
// Loading the next plane's operands one plane ahead needs ~40 more
// registers and measured slower.
constexpr int kAsmK = 31, kAsmJ = 8;

template <int LIM>
__global__ void __launch_bounds__(256, 4) k_assemble3(GridDev g, AsmParams a, const double* __restrict__ phi,
                                                      const double* __restrict__ phi_old, double* __restrict__ diag,
                                                      double* __restrict__ rhs_out, double* __restrict__ x0,
                                                      int planes) {
    __shared__ double rrN_s[2][kAsmJ][32];
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int kk = blockIdx.x * kAsmK + lane - 1;
    const int jj = blockIdx.y * kAsmJ + ty;
    const bool active = lane >= 1 && kk < n2 && jj < n1;
    const int i0 = blockIdx.z * planes;
    const int i1 = min(i0 + planes, n0);
    // loads of threads without a cell of their own stay in bounds: clamped
    // coordinates (lane 0 of the first tile keeps k = -1, a ghost cell, for
    // phi and its T face; face arrays of the other directions use k >= 0)
    const int jl = min(jj, n1 - 1);
    const int kl = min(kk, n2 - 1);
    const int kf = max(kl, 0);
    const int64_t n = a.dstride;
    const int64_t S0 = (int64_t)g.gn[1] * g.gn[2], S1 = g.gn[2];
    const int64_t nplane = (int64_t)n1 * n2;
    const int64_t jk = (int64_t)jl * n2 + kf;
    const int64_t fy_plane = (int64_t)(n1 + 1) * n2, fz_plane = (int64_t)n1 * (n2 + 1);
    // per-plane cursors (advanced by constant strides)
    const double* pc = phi + local_index(g, i0, jl, kl);
    const double* po = phi_old + local_index(g, i0, jl, kl);
    int64_t c = (int64_t)i0 * nplane + jk;
    int64_t fy_lo = (int64_t)i0 * fy_plane + (int64_t)jl * n2 + kf;
    int64_t fy_up = (int64_t)i0 * fy_plane + (int64_t)upper_face(g, 1, jl) * n2 + kf;
    int64_t fz_lo = (int64_t)i0 * fz_plane + (int64_t)jl * (n2 + 1) + kf;
    int64_t fz_up = (int64_t)i0 * fz_plane + (int64_t)jl * (n2 + 1) + (kl < 0 ? 0 : upper_face(g, 2, kl));

    double w0 = pc[-2 * S0], w1 = pc[-S0], w2 = pc[0], w3 = pc[S0], w4 = pc[2 * S0];
    double vx_lo = 0., Dx_lo = 0.;
    if (a.convection == 2) vx_lo = a.face_vel[0][(int64_t)i0 * nplane + jk];
    if (a.diffusion == 2) Dx_lo = a.face_D[0][(int64_t)i0 * nplane + jk];
    double rrW = 0.;
    if (a.convection) rrW = face_rr<LIM>(w0, w1, w2, w3, a.convection == 1 ? a.vel[0] : vx_lo);

    for (int i = i0; i < i1; i++) {
        const int buf = (i - i0) & 1;
        const int64_t fx_up = (int64_t)upper_face(g, 0, i) * nplane + jk;
        double coef[7];
#pragma unroll
        for (int p = 0; p < 7; p++) coef[p] = 0.;
        double rhs = 0.;

        if (a.dt > 0.) {                                   // DDT, weights (1, 1)
            const double tt = a.tt;
            coef[DARE_CENTER] = tt;
            rhs = 0. + tt * po[0];
        }

        if (a.convection) {                                // TVD * field, then divergence
            double vW, vEc, vSc, vNc, vB, vTc;
            if (a.convection == 1) {
                vW = vEc = a.vel[0];
                vSc = vNc = a.vel[1];
                vB = vTc = a.vel[2];
            } else {
                vW = vx_lo;
                vEc = a.face_vel[0][fx_up];
                vSc = a.face_vel[1][fy_lo];
                vNc = a.face_vel[1][fy_up];
                vTc = a.face_vel[2][fz_up];
                vB = __shfl_up_sync(0xFFFFFFFFu, vTc, 1);
            }
            const double ym1 = pc[-S1], yp1 = pc[S1], yp2 = pc[2 * S1];
            const double zm1 = pc[-1], zp1 = pc[1], zp2 = pc[2];
            const double rrE = face_rr<LIM>(w1, w2, w3, w4, vEc);
            const double rrN = face_rr<LIM>(ym1, w2, yp1, yp2, vNc);
            const double rrT = face_rr<LIM>(zm1, w2, zp1, zp2, vTc);
            rrN_s[buf][ty][lane] = rrN;
            const double rrB = __shfl_up_sync(0xFFFFFFFFu, rrT, 1);
            double rrS = 0.;
            if (ty == 0) rrS = face_rr<LIM>(pc[-2 * S1], ym1, w2, yp1, vSc);
            __syncthreads();
            if (ty > 0) rrS = rrN_s[buf][ty - 1][lane];

            double nb[7], cf[7], rr[7];
#pragma unroll
            for (int p = 0; p < 7; p++) nb[p] = cf[p] = rr[p] = 0.;
            {   // lower faces: nb = (vp v) 1, cf = (vn v) 1; upper faces: nb = (vn v) 1, cf = (vp v) 1,
                // vp = (v >= 0) in {0, 1}, vn = 1 - vp.  Evaluated without the
                // int -> double conversion: 1 * v = v (exactly; v >= 0 is never
                // NaN), 0 * v stays a multiplication (+-0, or NaN for v = +-inf),
                // and the trailing * 1 (also on the divergence terms) is the
                // identity on every value an arithmetic operation produces.
                const double vl[3] = {vW, vSc, vB}, vu[3] = {vEc, vNc, vTc};
                const double rl[3] = {rrW, rrS, rrB}, ru[3] = {rrE, rrN, rrT};
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int lo = 2 * d + 1, up = 2 * d + 2;
                    const bool lp = vl[d] >= 0., upp = vu[d] >= 0.;
                    const double l0 = 0. * vl[d], u0 = 0. * vu[d];
                    nb[lo] = lp ? vl[d] : l0;
                    cf[lo] = lp ? l0 : (1. * vl[d]);
                    rr[lo] = rl[d];
                    nb[up] = upp ? u0 : (1. * vu[d]);
                    cf[up] = upp ? vu[d] : u0;
                    rr[up] = ru[d];
                }
            }
            double sc[7];
            apply_divergence<3>(g, nb, cf, sc);
            if (a.scheme != DARE_SCHEME_EULER_BACKWARD) {     // s_c *= weight[0] (1: identity)
#pragma unroll
                for (int p = 0; p < 7; p++) sc[p] *= a.w[0];
            }
            double srhs = g.area[0] * (rr[DARE_EAST] - rr[DARE_WEST]);
            srhs += g.area[1] * (rr[DARE_NORTH] - rr[DARE_SOUTH]);
            srhs += g.area[2] * (rr[DARE_TOP] - rr[DARE_BOTTOM]);
            for (int t = 1; t <= a.nexp; t++) {                // explicit levels (copies of level 0)
                srhs += a.w[t] * g.area[0] * (rr[DARE_EAST] - rr[DARE_WEST]);
                srhs += a.w[t] * g.area[1] * (rr[DARE_NORTH] - rr[DARE_SOUTH]);
                srhs += a.w[t] * g.area[2] * (rr[DARE_TOP] - rr[DARE_BOTTOM]);
            }
#pragma unroll
            for (int p = 0; p < 7; p++) coef[p] += sc[p];       // MatrixBlock::Add
            rhs += srhs;
            rrW = rrE;
            vx_lo = vEc;
        }

        if (a.diffusion) {                                 // mb -= div(D, grad(mb))
            double Dlo[3], Dup[3];
            if (a.diffusion == 1) {
#pragma unroll
                for (int d = 0; d < 3; d++) Dlo[d] = Dup[d] = a.D;
            } else {
                Dlo[0] = Dx_lo;
                Dup[0] = a.face_D[0][fx_up];
                Dlo[1] = a.face_D[1][fy_lo];
                Dup[1] = a.face_D[1][fy_up];
                Dlo[2] = a.face_D[2][fz_lo];
                Dup[2] = a.face_D[2][fz_up];
                Dx_lo = Dup[0];
            }
            double nb[7], cf[7];
#pragma unroll
            for (int p = 0; p < 7; p++) nb[p] = cf[p] = 0.;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double dn = a.dn[d];
                const int lo = 2 * d + 1, up = 2 * d + 2;
                nb[lo] = (-dn) * Dlo[d];
                cf[lo] = dn * Dlo[d];
                nb[up] = dn * Dup[d];
                cf[up] = (-dn) * Dup[d];
            }
            double sc[7];
            apply_divergence<3>(g, nb, cf, sc);
            if (a.scheme != DARE_SCHEME_EULER_BACKWARD) {     // s_c *= weight[0] (1: identity)
#pragma unroll
                for (int p = 0; p < 7; p++) sc[p] *= a.w[0];
            }
#pragma unroll
            for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
            rhs += -1. * 0.;
        }

        if (active) {
            const int idx[3] = {i, jj, kk};
#pragma unroll
            for (int d = 0; d < 3; d++) {                  // boundary folding
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
            x0[c] = w2;
        }

        // advance one plane
        if (i + 1 < i1) {
            w0 = w1;
            w1 = w2;
            w2 = w3;
            w3 = w4;
            w4 = pc[3 * S0];
        }
        pc += S0;
        po += S0;
        c += nplane;
        fy_lo += fy_plane;
        fy_up += fy_plane;
        fz_lo += fz_plane;
        fz_up += fz_plane;
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
    a.tt = a.dt > 0. ? (g.volume * 1.) / a.dt : 0.;
    a.dstride = s->sdev.ncell;
    a.scheme = desc->scheme;
    a.nexp = scheme_weights(desc->scheme, a.w);
    if (a.nexp < 0) return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: unknown time scheme");
    for (int d = 0; d < 3; d++) a.dn[d] = 1. / g.dx[d];
    for (int d = 0; d < g.dim; d++) {
        if (a.diffusion == 2 && !a.face_D[d]) return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: face_D missing");
        if (a.convection == 2 && !a.face_vel[d])
            return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: face_vel missing");
    }
    if (a.diffusion < 0 || a.diffusion > 2 || a.convection < 0 || a.convection > 2 || a.limiter < 0 ||
        a.limiter > DARE_LIMITER_VANLEER)
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_assemble: bad descriptor");
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
    if (g.dim == 3) {
        // face-sharing kernel: blocks of 31 x 8 output cells (k, j), runs of
        // i-planes sized so the waves of resident blocks come out even
        static int resident = 0;
        if (!resident) {
            int occ = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_assemble3<DARE_LIMITER_VANLEER>, 32 * kAsmJ,
                                                              0) != cudaSuccess ||
                occ < 1)
                occ = 1;
            resident = occ * ctx->num_sms;
        }
        const int gx3 = (n2 + kAsmK - 1) / kAsmK, gy3 = (n1 + kAsmJ - 1) / kAsmJ;
        const int64_t units = (int64_t)gx3 * gy3;
        int best = n0;
        int64_t best_cost = INT64_MAX;
        for (int chunks = 1; chunks <= n0; chunks++) {
            const int pl = (n0 + chunks - 1) / chunks;
            if ((n0 + pl - 1) / pl != chunks) continue;
            const int64_t cost = ((units * chunks + resident - 1) / resident) * (pl + 2);
            if (cost < best_cost) {
                best_cost = cost;
                best = pl;
            }
        }
        const dim3 grid3(gx3, gy3, (unsigned)((n0 + best - 1) / best)), block3(32, kAsmJ, 1);
        // one launch per field component (its field values, its rows)
        for (int c = 0; c < s->ncomp; c++) {
            const double* pc = phi + (size_t)c * g.ncell_ghosted;
            const double* po = phi_old + (size_t)c * g.ncell_ghosted;
            double* dc = s->diag + (size_t)c * g.ncell;
            double* rc = s->rhs + (size_t)c * g.ncell;
            double* xc = s->x + (size_t)c * g.ncell;
            switch (a.limiter) {
#define DARE_ASM3(L)                                                                  \
    case L:                                                                           \
        k_assemble3<L><<<grid3, block3, 0, ctx->stream>>>(g, a, pc, po, dc, rc, xc, best); \
        break;
                DARE_ASM3(DARE_LIMITER_CDS)
                DARE_ASM3(DARE_LIMITER_UPWIND)
                DARE_ASM3(DARE_LIMITER_VANALBADA)
                DARE_ASM3(DARE_LIMITER_MINMOD)
                DARE_ASM3(DARE_LIMITER_VANLEER)
#undef DARE_ASM3
            }
            DARE_LAUNCHED(ctx);
        }
        return DARE_OK;
    }
    for (int c = 0; c < s->ncomp; c++) {
        const double* pc = phi + (size_t)c * g.ncell_ghosted;
        const double* po = phi_old + (size_t)c * g.ncell_ghosted;
        double* dc = s->diag + (size_t)c * g.ncell;
        double* rc = s->rhs + (size_t)c * g.ncell;
        double* xc = s->x + (size_t)c * g.ncell;
        if (g.dim == 2)
            k_assemble<2><<<grid, block, 0, ctx->stream>>>(g, a, pc, po, dc, rc, xc, planes);
        else
            k_assemble<1><<<grid, block, 0, ctx->stream>>>(g, a, pc, po, dc, rc, xc, planes);
        DARE_LAUNCHED(ctx);
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
