// dare_march.cuh -- device side of the BiCGStab(2) kernels: the scalar
// recurrences of BiCGStab2.inl, the fused stencil functors and the
// plane-marching stencil kernel they run in.
#pragma once

#include "dare_bicgstab2.cuh"

namespace dare_gpu {

// ---------------------------------------------------------------------------
// scalar recurrences, run by thread 0 of the last block of a kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ void finish(SolverState* st, int status, int step) {
    st->status = status;
    st->step = step;
    st->done = 1;
}

// Loop-top bookkeeping of the reference: `if (k > max_iteration) break;`,
// step (3) and step (4) given rho1 = <r_hat_0, r>.
__device__ inline void begin_iteration(SolverState* st, double rho1) {
    if (st->k > st->max_it) {
        finish(st, ST_MAXIT, 0);
        return;
    }
    st->rho0 = -st->omega2 * st->rho0;                       // (3)
    if (st->rho0 == 0.0) {
        finish(st, ST_BREAKDOWN, 3);
        return;
    }
    st->rho1 = rho1;                                         // (4)
    st->beta = st->alpha * st->rho1 / st->rho0;
    st->rho0 = st->rho1;
    if (st->rho0 == 0.0) finish(st, ST_BREAKDOWN, 4);
}

__device__ inline void finish_init(SolverState* st, const double* tot) {
    st->bnorm2 = tot[1];
    if (st->tol_relative) st->tol = st->tol * sqrt(tot[1]);
    st->rnorm0 = sqrt(tot[0]);
    st->rnorm = st->rnorm0;
    st->alpha = 0.;                                           // BiCGStab2.inl:182
    st->rho0 = st->omega1 = st->omega2 = 1.;                 // (1)
    st->k = 0;
    if (st->rnorm0 < st->tol) {                               // initial guess converged
        finish(st, ST_CONVERGED, 0);
        return;
    }
    if (isnan(st->rnorm0)) {
        finish(st, ST_NAN, 0);
        return;
    }
    st->k = 1;
    begin_iteration(st, tot[0]);                              // <r_hat_0, r> = <r, r>
}

__device__ inline void finish_gamma(SolverState* st, const double* tot, int step) {   // (7) / (14)
    st->gamma = tot[0];
    if (st->gamma == 0.0) {
        finish(st, ST_BREAKDOWN, step);
        return;
    }
    st->alpha = st->rho0 / st->gamma;
}

__device__ inline void finish_rho(SolverState* st, const double* tot) {               // (11)
    st->rho1 = tot[0];
    st->beta = st->alpha * st->rho1 / st->rho0;
    st->rho0 = st->rho1;
}

__device__ inline void finish_omega(SolverState* st, const double* tot) {             // (19)-(23)
    double omega_1 = tot[0], mu = tot[1], nu = tot[2], tau = tot[3], omega_2 = tot[4];
    if (mu == 0.) {
        finish(st, ST_BREAKDOWN, 20);
        return;
    }
    tau -= nu * nu / mu;                                      // (21)
    st->mu = mu;
    st->nu = nu;
    st->tau = tau;
    if (tau == 0.0) {
        finish(st, ST_TAU0, 21);
        return;
    }
    omega_2 = (omega_2 - (nu * omega_1) / mu) / tau;          // (22)
    omega_1 = (omega_1 - nu * omega_2) / mu;                  // (23)
    st->omega1 = omega_1;
    st->omega2 = omega_2;
}

__device__ inline void finish_update(SolverState* st, const double* tot) {            // (25) check, (3), (4)
    const double rnorm = sqrt(tot[0]);
    st->rnorm = rnorm;
    if (rnorm <= st->tol && st->k > 1) {
        finish(st, ST_CONVERGED, 0);
        return;
    }
    if (isnan(rnorm)) {
        finish(st, ST_NAN, 0);
        return;
    }
    st->k += 1;
    begin_iteration(st, tot[1]);
}

// ---------------------------------------------------------------------------
// fused stencil functors for the marching kernel
//   z(c):      the fused SpMV input at cell c
//   center():  everything done at the cell (writes, the SpMV row, dot terms)
//   done():    the scalar step, thread 0 of the last block
// ---------------------------------------------------------------------------
template <typename T, bool UNIT>
__device__ __forceinline__ T apply7(const OpT<T>& op, int64_t c, const T z[7]) {
    const int64_t n = op.n;
    T y = UNIT ? z[0] : op.c[c] * z[0];
    y += op.off[c] * z[1];
    y += op.off[n + c] * z[2];
    y += op.off[2 * n + c] * z[3];
    y += op.off[3 * n + c] * z[4];
    y += op.off[4 * n + c] * z[5];
    y += op.off[5 * n + c] * z[6];
    return y;
}

// K0: r = b - Op x; r_hat_0 = r; u = v = w = 0; sums <r,r>, <b,b>
template <typename T, bool UNIT>
struct FInit {
    using type = T;
    static constexpr int Q = 2;
    static constexpr bool kCheckDone = false;
    OpT<T> op;
    const T* x;
    const T* b;
    T *r, *rh, *u, *v, *w;
    __device__ void load(const SolverState*) {}
    __device__ T z(int64_t c) const { return x[c]; }
    __device__ void center(int64_t c, const T zz[7], double* acc) const {
        const T bc = b[c];
        const T rr = bc - apply7<T, UNIT>(op, c, zz);
        r[c] = rr;
        rh[c] = rr;
        u[c] = T(0);
        v[c] = T(0);
        w[c] = T(0);
        acc[0] += (double)rr * (double)rr;
        acc[1] += (double)bc * (double)bc;
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_init(st, tot); }
};

// K1: (5) u = r - beta u; (6) v = Op u; (7) gamma = <v, r_hat_0>
template <typename T, bool UNIT>
struct FStep1 {
    using type = T;
    static constexpr int Q = 1;
    static constexpr bool kCheckDone = true;
    OpT<T> op;
    const T *r, *u_in, *rh;
    T *u_out, *v;
    T beta;
    __device__ void load(const SolverState* st) { beta = (T)st->beta; }
    __device__ T z(int64_t c) const { return r[c] - beta * u_in[c]; }
    __device__ void center(int64_t c, const T zz[7], double* acc) const {
        u_out[c] = zz[0];
        const T vc = apply7<T, UNIT>(op, c, zz);
        v[c] = vc;
        acc[0] += (double)vc * (double)rh[c];
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_gamma(st, tot, 7); }
};

// K2: (8) r = r - alpha v; (9) s = Op r; (10) x = x + alpha u; (11) rho1 = <r_hat_0, s>
template <typename T, bool UNIT>
struct FStep2 {
    using type = T;
    static constexpr int Q = 1;
    static constexpr bool kCheckDone = true;
    OpT<T> op;
    const T *r_in, *v, *u, *rh;
    T *r_out, *s, *x;
    T alpha;
    __device__ void load(const SolverState* st) { alpha = (T)st->alpha; }
    __device__ T z(int64_t c) const { return -alpha * v[c] + r_in[c]; }
    __device__ void center(int64_t c, const T zz[7], double* acc) const {
        r_out[c] = zz[0];
        const T sc = apply7<T, UNIT>(op, c, zz);
        s[c] = sc;
        x[c] = alpha * u[c] + x[c];
        acc[0] += (double)rh[c] * (double)sc;
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_rho(st, tot); }
};

// K3: (12) v = s - beta v; (13) w = Op v; (14) gamma = <w, r_hat_0>
template <typename T, bool UNIT>
struct FStep3 {
    using type = T;
    static constexpr int Q = 1;
    static constexpr bool kCheckDone = true;
    OpT<T> op;
    const T *s, *v_in, *rh;
    T *v_out, *w;
    T beta;
    __device__ void load(const SolverState* st) { beta = (T)st->beta; }
    __device__ T z(int64_t c) const { return s[c] - beta * v_in[c]; }
    __device__ void center(int64_t c, const T zz[7], double* acc) const {
        v_out[c] = zz[0];
        const T wc = apply7<T, UNIT>(op, c, zz);
        w[c] = wc;
        acc[0] += (double)wc * (double)rh[c];
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_gamma(st, tot, 14); }
};

// K4: (15) u = r - beta u; (16) r = r - alpha v; (17) s = s - alpha w;
//     (18) t = Op s; (19)-(20) <r,s>, <s,s>, <s,t>, <t,t>, <r,t>; (21)-(23)
template <typename T, bool UNIT>
struct FStep4 {
    using type = T;
    static constexpr int Q = 5;
    static constexpr bool kCheckDone = true;
    OpT<T> op;
    T *u, *r;
    const T *v, *s_in, *w;
    T *s_out, *t;
    T alpha, beta;
    __device__ void load(const SolverState* st) {
        alpha = (T)st->alpha;
        beta = (T)st->beta;
    }
    __device__ T z(int64_t c) const { return -alpha * w[c] + s_in[c]; }
    __device__ void center(int64_t c, const T zz[7], double* acc) const {
        const T rc = r[c];
        u[c] = rc - beta * u[c];
        const T rn = -alpha * v[c] + rc;
        r[c] = rn;
        s_out[c] = zz[0];
        const T tc = apply7<T, UNIT>(op, c, zz);
        t[c] = tc;
        const double dr = rn, ds = zz[0], dt = tc;
        acc[0] += dr * ds;
        acc[1] += ds * ds;
        acc[2] += ds * dt;
        acc[3] += dt * dt;
        acc[4] += dr * dt;
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_omega(st, tot); }
};

// ||b - A x||^2 with a general operator, written to *out
template <typename T>
struct FResidual {
    using type = T;
    static constexpr int Q = 1;
    static constexpr bool kCheckDone = false;
    OpT<T> op;
    const T* x;
    const T* b;
    double* out;
    __device__ void load(const SolverState*) {}
    __device__ T z(int64_t c) const { return x[c]; }
    __device__ void center(int64_t c, const T zz[7], double* acc) const {
        const double r = (double)b[c] - (double)apply7<T, false>(op, c, zz);
        acc[0] += r * r;
    }
    __device__ void done(SolverState*, const double* tot) const { *out = sqrt(tot[0]); }
};

// Ahat[p][c] = A[p][c] * invd[neighbour_p(c)] (removed neighbours read 0)
struct FFold {
    using type = double;
    static constexpr int Q = 0;
    static constexpr bool kCheckDone = false;
    const double* diag;
    const double* invd;
    double* ahat;
    int64_t n;
    __device__ void load(const SolverState*) {}
    __device__ double z(int64_t c) const { return invd[c]; }
    __device__ void center(int64_t c, const double zz[7], double*) const {
#pragma unroll
        for (int p = 1; p < 7; p++) ahat[(p - 1) * n + c] = diag[p * n + c] * zz[p];
    }
    __device__ void done(SolverState*, const double*) const {}
};

// ---------------------------------------------------------------------------
// the plane-marching kernel
// ---------------------------------------------------------------------------
template <class K>
__global__ void __launch_bounds__(256) k_march(GridDev g, K kern, SolverState* st, double* partials, int chunk) {
    using T = typename K::type;
    if (K::kCheckDone && st->done) return;
    K k = kern;
    k.load(st);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* tile = reinterpret_cast<T*>(smem_raw);
    const int TK = blockDim.x, TJ = blockDim.y;
    const int W = TK + 2, H = TJ + 2;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int kk = blockIdx.x * TK + tx, jj = blockIdx.y * TJ + ty;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int i0 = blockIdx.z * chunk;
    const int i1 = min(i0 + chunk, n0);
    const bool inside = jj < n1 && kk < n2;
    const bool edge = jj <= n1 && kk <= n2;   // the first row / column past the grid is read as halo
    const int p0 = g.periodic[0], p1 = g.periodic[1], p2 = g.periodic[2];

    // fused input at (i, j, kx); wrapped on periodic dimensions, 0 outside
    auto Zat = [&](int i, int j, int kx) -> T {
        if (i < 0) {
            if (!p0) return T(0);
            i += n0;
        } else if (i >= n0) {
            if (!p0) return T(0);
            i -= n0;
        }
        if (j < 0) {
            if (!p1) return T(0);
            j += n1;
        } else if (j >= n1) {
            if (!p1) return T(0);
            j -= n1;
        }
        if (kx < 0) {
            if (!p2) return T(0);
            kx += n2;
        } else if (kx >= n2) {
            if (!p2) return T(0);
            kx -= n2;
        }
        if ((unsigned)i >= (unsigned)n0 || (unsigned)j >= (unsigned)n1 || (unsigned)kx >= (unsigned)n2) return T(0);
        return k.z(((int64_t)i * n1 + j) * n2 + kx);
    };

    double acc[K::Q > 0 ? K::Q : 1];
#pragma unroll
    for (int q = 0; q < (K::Q > 0 ? K::Q : 1); q++) acc[q] = 0.;
    T zprev = inside ? Zat(i0 - 1, jj, kk) : T(0);
    T zcur = edge ? Zat(i0, jj, kk) : T(0);
    int buf = 0;
    for (int i = i0; i < i1; i++) {
        const T znext = edge ? Zat(i + 1, jj, kk) : T(0);
        T* tb = tile + buf * W * H;
        tb[(ty + 1) * W + tx + 1] = zcur;
        if (inside) {
            if (ty == 0) tb[tx + 1] = Zat(i, jj - 1, kk);
            if (ty == TJ - 1) tb[(TJ + 1) * W + tx + 1] = Zat(i, jj + 1, kk);
            if (tx == 0) tb[(ty + 1) * W] = Zat(i, jj, kk - 1);
            if (tx == TK - 1) tb[(ty + 1) * W + TK + 1] = Zat(i, jj, kk + 1);
        }
        __syncthreads();
        if (inside) {
            const T z7[7] = {zcur, zprev, znext, tb[ty * W + tx + 1], tb[(ty + 2) * W + tx + 1],
                             tb[(ty + 1) * W + tx], tb[(ty + 1) * W + tx + 2]};
            k.center(((int64_t)i * n1 + jj) * n2 + kk, z7, acc);
        }
        zprev = zcur;
        zcur = znext;
        buf ^= 1;
    }
    if constexpr (K::Q > 0) {
        double tot[K::Q];
        if (!grid_reduce<K::Q>(acc, partials, &st->count, tot)) return;
        if (threadIdx.x == 0 && threadIdx.y == 0) k.done(st, tot);
    }
}

// K5: (24) x = x + w1 r + w2 s + alpha u; (25) r = r - w1 s - w2 t; ||r||;
//     u = u - w1 v - w2 w; then the next iteration's (3), (4).
template <typename T>
__global__ void __launch_bounds__(256) k_step5(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                               const T* __restrict__ s, const T* __restrict__ t,
                                               T* __restrict__ u, const T* __restrict__ v,
                                               const T* __restrict__ w, const T* __restrict__ rh,
                                               SolverState* st, double* partials) {
    if (st->done) return;
    const T w1 = (T)st->omega1, w2 = (T)st->omega2, alpha = (T)st->alpha;
    double acc[2] = {0., 0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const T rc = r[c], sc = s[c];
        T xc = w1 * rc + w2 * sc + x[c];
        xc = alpha * u[c] + xc;
        x[c] = xc;
        const T rn = -w1 * sc + -w2 * t[c] + rc;
        r[c] = rn;
        u[c] = -w1 * v[c] + -w2 * w[c] + u[c];
        acc[0] += (double)rn * (double)rn;
        acc[1] += (double)rh[c] * (double)rn;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) finish_update(st, tot);
}

static __global__ void k_invdiag(const double* __restrict__ dc, double* __restrict__ invd, int64_t n) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        invd[c] = 1. / dc[c];
}

// x = invd .* x (applyRightPrec at the end of the solve)
static __global__ void k_scale(int64_t n, const double* __restrict__ invd, double* __restrict__ x) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        x[c] = invd[c] * x[c];
}

template <class K>
inline int launch_march(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const K& kern, SolverState* st,
                        double* partials) {
    if (m.nblocks > kMaxBlocks) return set_error(ctx, DARE_ERR_UNSUPPORTED, "grid too large for the reduction");
    k_march<K><<<m.grid, m.block, m.smem, ctx->stream>>>(g, kern, st, partials, m.chunk);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

}  // namespace dare_gpu
