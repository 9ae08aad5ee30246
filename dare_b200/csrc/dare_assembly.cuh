// dare_assembly.cuh -- the assembly descriptor as the kernels see it, and the
// flux limiters of the TVD term (FluxLimiter.h:41-173, plus van Leer).
#pragma once

#include "dare_internal.cuh"

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
    // composition (MatrixBlock::Set / Add / operator-=): the sign each part
    // enters with (the fused descriptor: DDT +1, convection +1, diffusion -1),
    // whether the parts add to the coefficients already in the system, and
    // whether the boundary faces are folded at the end
    double sgn_ddt, sgn_conv, sgn_diff;
    int acc;
    int fold;
    // x ends the system shares with a neighbouring slab (bit 0 the low end,
    // bit 1 the high end): their faces are interior faces and stay unfolded
    int xint;
};

// Weights of the Divergence time schemes (TimeDiscretizationSchemes.h:29-76);
// returns the number of explicit levels, -1 for an unknown scheme.
inline int scheme_weights(int scheme, double w[3]) {
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

__device__ __forceinline__ int upper_face(const GridDev& g, int d, int i) {
    return (g.periodic[d] && i + 1 == g.n[d]) ? 0 : i + 1;
}

// The 3-D assembly (dare_assembly3.cu): one launch per field component, over
// the planes ib .. ie - 1 (ie < 0: through the last plane).
int launch_assemble3(dare_ctx* ctx, const GridDev& g, const AsmParams& a, const double* phi,
                     const double* phi_old, double* diag, double* rhs, double* x0, int ib = 0, int ie = -1);

}  // namespace dare_gpu
