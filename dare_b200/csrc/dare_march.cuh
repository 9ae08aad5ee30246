// dare_march.cuh -- device side of the BiCGStab(2) kernels: the scalar
// recurrences of BiCGStab2.inl, the fused stencil functors and the
// plane-marching stencil kernel they run in.
//
// The marching kernel is persistent: one grid of (blocks per SM x SMs)
// blocks pulls equal work items -- a (j,k) tile and a run of i-planes -- from
// a device queue.  Inside an item the block walks along i.  Every plane is
// staged in shared memory by asynchronous copies (cp.async): the inputs of the
// fused SpMV operand with a one-cell j/k halo, and the per-cell streams of the
// centre step (coefficients, vectors).  A ring of three stages keeps the
// copies of planes i+1 and i+2 in flight while plane i computes, so HBM
// latency hides behind the arithmetic without holding data in registers.
// Dot-product partials are kept per item and summed in item order by the
// last item, so results do not depend on which block took which item.
#pragma once

#include <type_traits>

#include "dare_bicgstab2.cuh"

namespace dare_gpu {

// ---------------------------------------------------------------------------
// scalar recurrences, run by thread 0 of the block that finishes last
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
    if (step == 7) st->alpha1 = st->alpha;   // the alpha of step (10), applied in the last kernel
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
// operator rows: p[0..5] = W,E,S,N,B,T off-diagonals, p[6] = centre (general
// operator only); z[0..6] = C,W,E,S,N,B,T values of the SpMV operand
// ---------------------------------------------------------------------------
template <bool UNIT>
struct NCoef {
    static constexpr int value = UNIT ? 6 : 7;
};

template <typename T, bool UNIT>
__device__ __forceinline__ T apply_pre(const T* p, const T (&z)[7]) {
    T y = UNIT ? z[0] : p[6] * z[0];
    y += p[0] * z[1];
    y += p[1] * z[2];
    y += p[2] * z[3];
    y += p[3] * z[4];
    y += p[4] * z[5];
    y += p[5] * z[6];
    return y;
}

template <typename T, bool UNIT, int NP>
__host__ __device__ inline void set_coef_streams(const OpT<T>& op, const T* (&ps)[NP]) {
#pragma unroll
    for (int q = 0; q < 6; q++) ps[q] = op.off + q * op.n;
    if (!UNIT) ps[6] = op.c;
}

// ---------------------------------------------------------------------------
// fused stencil functors (plain data, built on the host)
//   zs[NZ] / zc(a, b):   the SpMV operand z = zc(zs[0][c], zs[1][c])
//   ps[NP]:              per-cell streams staged for the centre step
//   center(c, z, p, acc): writes, the SpMV row, dot-product terms
//   done(st, tot):       the scalar step, by the block finishing the last item
// ---------------------------------------------------------------------------

// K0: r = b - Op x; r_hat_0 = r; u = 0; sums <r,r>, <b,b>.  (The reference
// also zeroes v and w in step (1); every iteration writes both before it
// reads them -- v in step (6), w in step (13) -- so they are left alone.)
template <typename T, bool UNIT>
struct FInit {
    using type = T;
    static constexpr int Q = 2, NZ = 1, NC = NCoef<UNIT>::value, NP = NC + 1;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;   // two cells per thread (see launch_march)
    const T* zs[2];   // x
    const T* ps[NP];  // coefficients, b
    T *r, *rh, *u;
    __device__ void load(const SolverState*) {}
    __device__ T zc(T a, T) const { return a; }
    __device__ void center(int64_t c, const T (&zz)[7], const T* p, double* acc) const {
        const T bc = p[NC];
        const T rr = bc - apply_pre<T, UNIT>(p, zz);
        r[c] = rr;
        rh[c] = rr;
        u[c] = T(0);
        acc[0] += (double)rr * (double)rr;
        acc[1] += (double)bc * (double)bc;
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_init(st, tot); }
};

// K1: (5) u = r - beta u; (6) v = Op u; (7) gamma = <v, r_hat_0>
template <typename T, bool UNIT>
struct FStep1 {
    using type = T;
    static constexpr int Q = 1, NZ = 2, NC = NCoef<UNIT>::value, NP = NC + 1;
    static constexpr bool kCheckDone = true;
    static constexpr bool kPairs = sizeof(T) == 4;   // two cells per thread (see launch_march)
    const T* zs[2];   // r, u
    const T* ps[NP];  // coefficients, r_hat_0
    T *u_out, *v;
    T beta;
    __device__ void load(const SolverState* st) { beta = (T)st->beta; }
    __device__ T zc(T r, T u) const { return r - beta * u; }
    __device__ void center(int64_t c, const T (&zz)[7], const T* p, double* acc) const {
        u_out[c] = zz[0];
        const T vc = apply_pre<T, UNIT>(p, zz);
        v[c] = vc;
        acc[0] += (double)vc * (double)p[NC];
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_gamma(st, tot, 7); }
};

// K2: (8) r = r - alpha v; (9) s = Op r; (11) rho1 = <r_hat_0, s>.  Step
// (10), x = x + alpha u, waits for K5 (x is read by nothing in between and
// step (15) leaves this u in place), which saves x's read and write here.
template <typename T, bool UNIT>
struct FStep2 {
    using type = T;
    static constexpr int Q = 1, NZ = 2, NC = NCoef<UNIT>::value, NP = NC + 1;
    static constexpr bool kCheckDone = true;
    static constexpr bool kPairs = sizeof(T) == 4;   // two cells per thread (see launch_march)
    const T* zs[2];   // v, r
    const T* ps[NP];  // coefficients, r_hat_0
    T *r_out, *s;
    T alpha;
    __device__ void load(const SolverState* st) { alpha = (T)st->alpha; }
    __device__ T zc(T v, T r) const { return -alpha * v + r; }
    __device__ void center(int64_t c, const T (&zz)[7], const T* p, double* acc) const {
        r_out[c] = zz[0];
        const T sc = apply_pre<T, UNIT>(p, zz);
        s[c] = sc;
        acc[0] += (double)p[NC] * (double)sc;
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_rho(st, tot); }
};

// K3: (12) v = s - beta v; (13) w = Op v; (14) gamma = <w, r_hat_0>
template <typename T, bool UNIT>
struct FStep3 {
    using type = T;
    static constexpr int Q = 1, NZ = 2, NC = NCoef<UNIT>::value, NP = NC + 1;
    static constexpr bool kCheckDone = true;
    static constexpr bool kPairs = sizeof(T) == 4;   // two cells per thread (see launch_march)
    const T* zs[2];   // s, v
    const T* ps[NP];  // coefficients, r_hat_0
    T *v_out, *w;
    T beta;
    __device__ void load(const SolverState* st) { beta = (T)st->beta; }
    __device__ T zc(T s, T v) const { return s - beta * v; }
    __device__ void center(int64_t c, const T (&zz)[7], const T* p, double* acc) const {
        v_out[c] = zz[0];
        const T wc = apply_pre<T, UNIT>(p, zz);
        w[c] = wc;
        acc[0] += (double)wc * (double)p[NC];
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_gamma(st, tot, 14); }
};

// K4: (16) r = r - alpha v; (17) s = s - alpha w; (18) t = Op s;
//     (19)-(20) <r,s>, <s,s>, <s,t>, <t,t>, <r,t>; (21)-(23).  The new r
//     goes to the other r buffer, so K5 can still form step (15)'s
//     u = r - beta u from this kernel's input r.
template <typename T, bool UNIT>
struct FStep4 {
    using type = T;
    static constexpr int Q = 5, NZ = 2, NC = NCoef<UNIT>::value, NP = NC + 2;
    static constexpr bool kCheckDone = true;
    static constexpr bool kPairs = sizeof(T) == 4;   // two cells per thread (see launch_march)
    const T* zs[2];   // w, s
    const T* ps[NP];  // coefficients, r (of step (8)), v
    T *r_out, *s_out, *t;
    T alpha;
    __device__ void load(const SolverState* st) { alpha = (T)st->alpha; }
    __device__ T zc(T w, T s) const { return -alpha * w + s; }
    __device__ void center(int64_t c, const T (&zz)[7], const T* p, double* acc) const {
        const T rn = -alpha * p[NC + 1] + p[NC];
        r_out[c] = rn;
        s_out[c] = zz[0];
        const T tc = apply_pre<T, UNIT>(p, zz);
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

// ||b - A x||_2 with the general operator, written to *out
template <typename T>
struct FResidual {
    using type = T;
    static constexpr int Q = 1, NZ = 1, NP = 8;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;   // two cells per thread (see launch_march)
    const T* zs[2];   // x
    const T* ps[NP];  // 7 coefficients, b
    double* out;
    __device__ void load(const SolverState*) {}
    __device__ T zc(T a, T) const { return a; }
    __device__ void center(int64_t, const T (&zz)[7], const T* p, double* acc) const {
        const double r = (double)p[7] - (double)apply_pre<T, false>(p, zz);
        acc[0] += r * r;
    }
    __device__ void done(SolverState*, const double* tot) const { *out = sqrt(tot[0]); }
};

// Ahat[q][c] = A[q][c] * invd[neighbour_q(c)] (removed neighbours read 0)
struct FFold {
    using type = double;
    static constexpr int Q = 0, NZ = 1, NP = 6;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;   // two cells per thread (see launch_march)
    const double* zs[2];   // invd
    const double* ps[NP];  // the 6 off-diagonals of A
    double* ahat;
    int64_t n;
    __device__ void load(const SolverState*) {}
    __device__ double zc(double a, double) const { return a; }
    __device__ void center(int64_t c, const double (&zz)[7], const double* p, double*) const {
#pragma unroll
        for (int q = 0; q < 6; q++) ahat[q * n + c] = p[q] * zz[q + 1];
    }
    __device__ void done(SolverState*, const double*) const {}
};

// The same, rounded to FP32: the operator of the FP32 inner solves, written
// without an FP64 copy
struct FFold32 {
    using type = double;
    static constexpr int Q = 0, NZ = 1, NP = 6;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;   // two cells per thread (see launch_march)
    const double* zs[2];   // invd
    const double* ps[NP];  // the 6 off-diagonals of A
    float* ahat;
    int64_t n;
    __device__ void load(const SolverState*) {}
    __device__ double zc(double a, double) const { return a; }
    __device__ void center(int64_t c, const double (&zz)[7], const double* p, double*) const {
#pragma unroll
        for (int q = 0; q < 6; q++) ahat[q * n + c] = (float)(p[q] * zz[q + 1]);
    }
    __device__ void done(SolverState*, const double*) const {}
};

// K0 with the Jacobi fold, one pass instead of FFold then FInit: Ahat[q][c] =
// A[q][c] * invd[neighbour_q(c)] written, then r = b - Ahat y from those
// values, r_hat_0 = r, u = 0; sums <r,r>, <b,b>.  The products and sums are
// the two kernels' own, in their order, so the results are the same bits.
// Split operands (kSplit): the kernel hands over both staged arrays' seven
// values, invd and y, instead of one combined operand.
struct FFoldInit {
    using type = double;
    static constexpr int Q = 2, NZ = 2, NP = 7;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;
    static constexpr bool kSplit = true;
    const double* zs[2];   // invd, y
    const double* ps[NP];  // the 6 off-diagonals of A, b
    double *ahat, *r, *rh, *u;
    int64_t n;
    __device__ void load(const SolverState*) {}
    __device__ double zc(double a, double) const { return a; }   // (the combined operand is not used)
    __device__ void center2(int64_t c, const double (&iv)[7], const double (&y)[7], const double* p,
                            double* acc) const {
        double a[6];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            a[q] = p[q] * iv[q + 1];
            ahat[q * n + c] = a[q];
        }
        double yy = y[0];   // apply_pre<double, true>(a, y)
        yy += a[0] * y[1];
        yy += a[1] * y[2];
        yy += a[2] * y[3];
        yy += a[3] * y[4];
        yy += a[4] * y[5];
        yy += a[5] * y[6];
        const double bc = p[6];
        const double rr = bc - yy;
        r[c] = rr;
        rh[c] = rr;
        u[c] = 0.;
        acc[0] += rr * rr;
        acc[1] += bc * bc;
    }
    __device__ void done(SolverState* st, const double* tot) const { finish_init(st, tot); }
};

template <class K, class = void>
struct SplitOperands {
    static constexpr bool value = false;
};
template <class K>
struct SplitOperands<K, std::void_t<decltype(K::kSplit)>> {
    static constexpr bool value = K::kSplit;
};

// ---------------------------------------------------------------------------
// the functors of the init kernel and of one iteration over the vectors vs
// (halves a of r / u current, b = 1 - a written), shared by the single-grid
// and the slab drivers
// ---------------------------------------------------------------------------
template <typename T, bool UNIT>
FInit<T, UNIT> make_init(const OpT<T>& op, const VecsT<T>& vs) {
    using F = FInit<T, UNIT>;
    F f{};
    f.zs[0] = vs.x;
    set_coef_streams<T, UNIT, F::NP>(op, f.ps);
    f.ps[F::NC] = vs.b;
    f.r = vs.r[0];
    f.rh = vs.rh;
    f.u = vs.u[0];
    return f;
}
template <typename T, bool UNIT>
FStep1<T, UNIT> make_step1(const OpT<T>& op, const VecsT<T>& vs) {
    FStep1<T, UNIT> f{};
    f.zs[0] = vs.r[0];
    f.zs[1] = vs.u[0];
    set_coef_streams<T, UNIT, FStep1<T, UNIT>::NP>(op, f.ps);
    f.ps[NCoef<UNIT>::value] = vs.rh;
    f.u_out = vs.u[1];
    f.v = vs.v[0];
    return f;
}
template <typename T, bool UNIT>
FStep2<T, UNIT> make_step2(const OpT<T>& op, const VecsT<T>& vs) {
    constexpr int NC = NCoef<UNIT>::value;
    FStep2<T, UNIT> f{};
    f.zs[0] = vs.v[0];
    f.zs[1] = vs.r[0];
    set_coef_streams<T, UNIT, FStep2<T, UNIT>::NP>(op, f.ps);
    f.ps[NC] = vs.rh;
    f.r_out = vs.r[1];
    f.s = vs.s[0];
    return f;
}
template <typename T, bool UNIT>
FStep3<T, UNIT> make_step3(const OpT<T>& op, const VecsT<T>& vs) {
    FStep3<T, UNIT> f{};
    f.zs[0] = vs.s[0];
    f.zs[1] = vs.v[0];
    set_coef_streams<T, UNIT, FStep3<T, UNIT>::NP>(op, f.ps);
    f.ps[NCoef<UNIT>::value] = vs.rh;
    f.v_out = vs.v[1];
    f.w = vs.w;
    return f;
}
template <typename T, bool UNIT>
FStep4<T, UNIT> make_step4(const OpT<T>& op, const VecsT<T>& vs) {
    constexpr int NC = NCoef<UNIT>::value;
    FStep4<T, UNIT> f{};
    f.zs[0] = vs.w;
    f.zs[1] = vs.s[0];
    set_coef_streams<T, UNIT, FStep4<T, UNIT>::NP>(op, f.ps);
    f.ps[NC] = vs.r[1];
    f.ps[NC + 1] = vs.v[1];
    f.r_out = vs.r[0];
    f.s_out = vs.s[1];
    f.t = vs.t;
    return f;
}
inline FResidual<double> make_residual(const OpT<double>& op, const double* x, const double* b, double* out) {
    FResidual<double> f{};
    f.zs[0] = x;
    set_coef_streams<double, false, 8>(op, f.ps);
    f.ps[7] = b;
    f.out = out;
    return f;
}
inline FFold make_fold(const double* diag, const double* invd, double* ahat, int64_t n) {
    FFold f{};
    f.zs[0] = invd;
    for (int q = 0; q < 6; q++) f.ps[q] = diag + (q + 1) * n;
    f.ahat = ahat;
    f.n = n;
    return f;
}

// ---------------------------------------------------------------------------
// item reduction: partials are indexed by item; the item whose counter
// increment completes the set sums them in item order.
// ---------------------------------------------------------------------------
template <int Q>
__device__ bool item_reduce(double (&v)[Q], double* __restrict__ partials, int item, int nitems,
                            unsigned int* counter, double (&tot)[Q]) {
    __shared__ double sh[32 * kMaxQ];
    __shared__ bool is_last;
    block_sum<Q>(v, sh);
    const int tid = thread_linear();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) partials[q * kMaxBlocks + item] = v[q];
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        is_last = (prev == (unsigned)nitems - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double a[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) a[q] = 0.;
    const int nt = blockDim.x * blockDim.y;
    for (int b = tid; b < nitems; b += nt) {
#pragma unroll
        for (int q = 0; q < Q; q++) a[q] += __ldcg(partials + q * kMaxBlocks + b);
    }
    block_sum<Q>(a, sh);
#pragma unroll
    for (int q = 0; q < Q; q++) tot[q] = a[q];
    if (tid == 0) *counter = 0u;
    return true;
}

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies (zero-filled when src_bytes == 0)
// ---------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int src = valid ? BYTES : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Shared-memory elements of one stage of a marching block for functor K: a
// tile of tw x tj cells (tw = threads in x times cells per thread), operand
// rows padded by ic columns on each side (the halo column sits at ic - 1 and
// ic + tw), plus the per-cell streams.
template <class K>
__host__ __device__ constexpr size_t march_stage_elems(int tw, int tj, int ic) {
    return (size_t)K::NZ * (tw + 2 * ic) * (tj + 2) + (size_t)K::NP * tw * tj;
}
template <class K>
inline size_t march_smem_bytes(const MarchCfg& m) {
    const int ic = m.cpt;   // first interior column: one row segment of padding
    return 3 * march_stage_elems<K>(m.block.x * m.cpt, m.block.y, ic) * sizeof(typename K::type);
}

// two consecutive elements of shared memory in one load (16-byte aligned for
// double, 8-byte for float)
template <typename T>
struct Pair {
    T x, y;
};
template <typename T>
__device__ __forceinline__ Pair<T> ld_pair(const T* p) {
    if constexpr (sizeof(T) == 8) {
        const double2 v = *reinterpret_cast<const double2*>(p);
        return Pair<T>{(T)v.x, (T)v.y};
    } else {
        const float2 v = *reinterpret_cast<const float2*>(p);
        return Pair<T>{(T)v.x, (T)v.y};
    }
}

// ---------------------------------------------------------------------------
// the persistent plane-marching kernel.  CPT cells per thread along k: with
// CPT = 2 (even n2) every staged row segment of a thread is one 16-byte copy
// (8 bytes for FP32), halving the per-cell copies, index arithmetic and
// barrier waits; the operand rows are padded so those copies stay aligned.
// ---------------------------------------------------------------------------
// Register budgets, measured at 256^3: two cells per thread held to 80
// registers (steps 1 and 3: 0.264 -> 0.257 ms); one cell per thread up to 128,
// two blocks per SM (held to 80 registers, steps 2 and 4 went from
// 0.343 / 0.353 ms to 0.408 / 0.433 ms, also when the maximum shared-memory
// carveout then let three blocks in; that carveout also slowed steps 1 and 3
// to 0.354 ms, so the default carveout stays).
// HALO (slabs): the planes before the first and after the last plane of the
// grid come from m.halo when set.
// Blocks per SM the register budget is set for: three (80 registers) with
// two cells per thread, two (128) with one.  Step 4 (two staged operands,
// eight streams, five FP64 dot products) takes two blocks of 128 registers
// with two cells per thread too: held to 80, the FP32 step 4 of the
// refinement ran 1.66 ms at 512^3 (64 % of copy bandwidth), with 128
// registers 1.18 ms (90 %).
template <class K, int CPT>
struct MarchMinBlocks {
    static constexpr int value = CPT == 2 ? 3 : 2;
};
template <typename T, bool UNIT, int CPT>
struct MarchMinBlocks<FStep4<T, UNIT>, CPT> {
    static constexpr int value = 2;
};

template <class K, int CPT = 1, bool HALO = false, bool PAIR = false>
__global__ void __launch_bounds__(256, MarchMinBlocks<K, CPT>::value) k_march(GridDev g, K kern, SolverState* st, double* partials,
                                                                   MarchCfg m) {
    using T = typename K::type;
    constexpr int NZ = K::NZ, NP = K::NP;
    constexpr int QA = K::Q > 0 ? K::Q : 1;
    constexpr int VEC = 16 / (int)sizeof(T);    // cells of one 16-byte copy
    static_assert(!PAIR || VEC % CPT == 0, "16-byte staging: a copy covers whole thread segments");
    constexpr int IC = PAIR ? VEC : CPT;        // first interior column of a staged operand row
    constexpr int CB = CPT * (int)sizeof(T);    // bytes of one thread's row segment
    if (K::kCheckDone && st->done) return;
    K k = kern;
    k.load(st);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    __shared__ int s_item;
    const int TK = blockDim.x, TJ = blockDim.y;
    const int TW = TK * CPT;                    // tile width in cells
    const int W = TW + 2 * IC, H = TJ + 2;
    const int ZT = W * H;                       // one staged operand tile
    const int NCT = TW * TJ;                    // cells of the tile
    const int STAGE = NZ * ZT + NP * NCT;       // elements per stage
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + TK * ty;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int n0c = n0 / g.ncomp;               // planes of one field component
    const int p0 = g.periodic[0], p1 = g.periodic[1], p2 = g.periodic[2];
    const int64_t plane = (int64_t)n1 * n2;
    const int tiles = m.tiles_x * m.tiles_y;

    // Geometry of one work item for this thread.
    struct Geo {
        int i0, i1;
        int cb;        // first stacked plane of this item's component
        bool inside, hS, hN, hB, hT;
        int64_t o_c, o_s, o_n, o_b, o_t, o_own;
        int64_t o_pair;   // PAIR: in-plane offset of this thread's pair of stream cells (-1: outside)
        int64_t o_op;     // PAIR: in-plane offset of this thread's operand copy (-1: zero)
    };
    // PAIR: every value staged as part of a 16-byte copy of VEC cells (FP64
    // with one cell per thread, FP32 with two: row length and tile width
    // multiples of VEC).  The per-cell streams: the first half of the threads
    // copies the even-numbered streams and the second half the odd ones, one
    // 16-byte copy each -- half the copies and address arithmetic of one
    // copy per thread and stream (256^3 FP64 step 4: 0.316 -> 0.298 ms).
    static_assert(!PAIR || VEC / CPT == 2, "16-byte staging: two thread sets");
    const int npairs = NCT / VEC;               // 16-byte copies per stream and plane (half the threads)
    const int par = tid >= npairs;
    const int e_pair = tid - par * npairs;
    const int hw = TW / VEC > 0 ? TW / VEC : 1;   // copies per row (PAIR needs TW % VEC == 0)
    const int pr_row = e_pair / hw, pr_col = VEC * (e_pair - pr_row * hw);
    // PAIR: the operand tiles' rows 0 .. TJ+1 (j0-1 .. j0+TJ) as 16-byte copies,
    // then the single halo cells k0-1 and k0+TW of rows 1 .. TJ; thread tid
    // makes one copy of every operand array (op_kind 2: 16 bytes, 1: one
    // cell, 0: none) -- (TJ+2) TW/VEC + 2 TJ copies, all threads alike, in place
    // of one copy per cell plus the halo copies of the edge threads (256^3
    // FP64 step 4: 0.298 -> 0.285 ms, 6.1 TB/s; the FP32 kernels on 64 x 8
    // tiles run two cells per thread this way, 512^3 FP32-refine solve 52.8
    // -> 51.7 ms)
    int op_kind = 0, op_row = 0, op_col = 0, op_dk = 0;
    if constexpr (PAIR) {
        const int npr = (TJ + 2) * hw;
        if (tid < npr) {
            op_kind = 2;
            op_row = tid / hw;
            op_dk = VEC * (tid - op_row * hw);
            op_col = IC + op_dk;
        } else if (tid < npr + 2 * TJ) {
            const int e = tid - npr;
            op_kind = 1;
            op_row = 1 + (e >> 1);
            op_dk = (e & 1) ? TW : -1;
            op_col = IC + op_dk;
        }
    }
    // in-plane position (j, kx) -> wrapped offset, or -1 when outside (zero)
    auto jk_offset = [&](int j, int kx) -> int64_t {
        if (j < 0) {
            if (!p1) return -1;
            j += n1;
        } else if (j >= n1) {
            if (!p1) return -1;
            j -= n1;
        }
        if (kx < 0) {
            if (!p2) return -1;
            kx += n2;
        } else if (kx >= n2) {
            if (!p2) return -1;
            kx -= n2;
        }
        if ((unsigned)j >= (unsigned)n1 || (unsigned)kx >= (unsigned)n2) return -1;
        return (int64_t)j * n2 + kx;
    };
    auto geometry = [&](int item) {
        Geo G;
        const int tile_id = item % tiles;
        const int chunk = item / tiles;
        const int kk = (tile_id % m.tiles_x) * TW + CPT * tx;   // this thread's first cell
        const int jj = (tile_id / m.tiles_x) * TJ + ty;
        // runs of planes never cross from one field component to the next
        const int comp = g.ncomp > 1 ? chunk / m.cpc : 0;
        G.cb = comp * n0c;
        G.i0 = G.cb + (chunk - comp * m.cpc) * m.planes;
        G.i1 = min(G.i0 + m.planes, G.cb + n0c);
        // (n2 is even when CPT = 2, so a thread's cells are both inside or both outside)
        G.inside = jj < n1 && kk < n2;
        const bool edge = jj <= n1 && kk <= n2;   // the first row / column past the grid is read as halo
        G.hS = G.inside && ty == 0;
        G.hN = G.inside && ty == TJ - 1;
        G.hB = G.inside && tx == 0;
        G.hT = G.inside && tx == TK - 1;
        G.o_c = edge ? jk_offset(jj, kk) : -1;
        G.o_s = G.hS ? jk_offset(jj - 1, kk) : -1;
        G.o_n = G.hN ? jk_offset(jj + 1, kk) : -1;
        G.o_b = G.hB ? jk_offset(jj, kk - 1) : -1;
        G.o_t = G.hT ? jk_offset(jj, kk + CPT) : -1;
        G.o_own = G.inside ? (int64_t)jj * n2 + kk : 0;
        G.o_pair = G.o_op = -1;
        if constexpr (PAIR) {
            const int tj0 = (tile_id / m.tiles_x) * TJ, tk0 = (tile_id % m.tiles_x) * TW;
            const int pj = tj0 + pr_row, pk = tk0 + pr_col;
            G.o_pair = (pj < n1 && pk < n2) ? (int64_t)pj * n2 + pk : -1;
            // a pair past n2 starts at the wrapped (or removed) first cell; its
            // second cell is never read
            if (op_kind) G.o_op = jk_offset(tj0 - 1 + op_row, tk0 + op_dk);
        }
        return G;
    };
    auto slot_of = [&](const Geo& G, int p) { return (p - G.i0 + 1) % 3; };
    // Stage plane p into its ring slot: operand inputs with halo, and (when
    // `full`) the per-cell streams.  Out-of-range planes are zeros.
    auto stage = [&](const Geo& G, int p, bool full) {
        T* sb = smem + (size_t)slot_of(G, p) * STAGE;
        bool pv = true;
        int pp = p - G.cb;   // plane within the component, wrapped on a periodic x
        if (pp < 0) {
            pv = p0;
            pp += n0c;
        } else if (pp >= n0c) {
            pv = p0;
            pp -= n0c;
        }
        const int64_t base = (int64_t)(G.cb + pp) * plane;
        const int col = IC + CPT * tx;
#pragma unroll
        for (int z = 0; z < NZ; z++) {
            const T* src = k.zs[z];
            T* zt = sb + z * ZT;
            int64_t zb = base;
            bool zv = pv;
            if constexpr (HALO) {
                const int hside = p - G.cb < 0 ? 0 : (p - G.cb >= n0c ? 1 : -1);   // a plane past the slab
                if (hside >= 0 && m.halo[z][hside]) {   // the neighbour's plane, exchanged into a local buffer
                    src = static_cast<const T*>(m.halo[z][hside]) + (int64_t)(G.cb / n0c) * plane;   // [component][plane]
                    zb = 0;
                    zv = true;
                }
            }
            if constexpr (PAIR) {
                if (op_kind == 2)
                    cp_async<16>(zt + op_row * W + op_col, src + zb + (G.o_op < 0 ? 0 : G.o_op), zv && G.o_op >= 0);
                else if (op_kind == 1)
                    cp_async<(int)sizeof(T)>(zt + op_row * W + op_col, src + zb + (G.o_op < 0 ? 0 : G.o_op),
                                             zv && G.o_op >= 0);
                continue;
            }
            cp_async<CB>(zt + (ty + 1) * W + col, src + zb + (G.o_c < 0 ? 0 : G.o_c), zv && G.o_c >= 0);
            if (G.hS) cp_async<CB>(zt + col, src + zb + (G.o_s < 0 ? 0 : G.o_s), zv && G.o_s >= 0);
            if (G.hN)
                cp_async<CB>(zt + (TJ + 1) * W + col, src + zb + (G.o_n < 0 ? 0 : G.o_n), zv && G.o_n >= 0);
            if (G.hB)
                cp_async<sizeof(T)>(zt + (ty + 1) * W + IC - 1, src + zb + (G.o_b < 0 ? 0 : G.o_b),
                                    zv && G.o_b >= 0);
            if (G.hT)
                cp_async<sizeof(T)>(zt + (ty + 1) * W + IC + TW, src + zb + (G.o_t < 0 ? 0 : G.o_t),
                                    zv && G.o_t >= 0);
        }
        if constexpr (PAIR) {
            if (full) {
                T* pt = sb + NZ * ZT + pr_row * TW + pr_col;
#pragma unroll
                for (int q = 0; q < NP; q++)
                    if ((q & 1) == par)
                        cp_async<16>(pt + q * NCT, k.ps[q] + base + (G.o_pair < 0 ? 0 : G.o_pair), G.o_pair >= 0);
            }
            return;
        }
        if (full && G.inside) {
            T* pt = sb + NZ * ZT + ty * TW + CPT * tx;
#pragma unroll
            for (int q = 0; q < NP; q++) cp_async<CB>(pt + q * NCT, k.ps[q] + base + G.o_own, true);
        }
    };
    // prologue of an item: planes i0-1 (operand only), i0, i0+1
    auto prologue = [&](const Geo& G) {
        stage(G, G.i0 - 1, false);
        cp_async_commit();
        stage(G, G.i0, true);
        cp_async_commit();
        stage(G, G.i0 + 1, G.i0 + 1 < G.i1);
        cp_async_commit();
    };
    auto zval = [&](const T* sb, int row, int col) -> T {
        const T a = sb[row * W + col];
        const T b = NZ > 1 ? sb[ZT + row * W + col] : T(0);
        return k.zc(a, b);
    };

    // Items come from the queue one ahead: the next index is fetched when an
    // item starts, and the next item's prologue copies are issued before the
    // current item's reduction, so the queue atomic, the reduction and the
    // first planes' DRAM latency overlap.
    __shared__ int s_next;
    if (tid == 0) s_item = (int)atomicAdd(&st->queue, 1u);
    __syncthreads();
    int item = s_item;
    Geo G = geometry(item < m.nitems ? item : 0);
    if (item < m.nitems) prologue(G);
    while (item < m.nitems) {
        if (tid == 0) s_next = (int)atomicAdd(&st->queue, 1u);
        double acc[QA];
#pragma unroll
        for (int q = 0; q < QA; q++) acc[q] = 0.;
        cp_async_wait<2>();
        __syncthreads();
        constexpr bool SPLIT = SplitOperands<K>::value;
        T zprev[CPT];
        T zprev_b = T(0);   // split operands: the second array's value at plane i - 1
        if constexpr (SPLIT) {
            const T* s0 = smem + (size_t)slot_of(G, G.i0 - 1) * STAGE + (ty + 1) * W + IC + tx;
            zprev[0] = G.inside ? s0[0] : T(0);
            zprev_b = G.inside ? s0[ZT] : T(0);
        } else {
#pragma unroll
            for (int c = 0; c < CPT; c++)
                zprev[c] =
                    G.inside ? zval(smem + (size_t)slot_of(G, G.i0 - 1) * STAGE, ty + 1, IC + CPT * tx + c) : T(0);
        }
        __syncthreads();
        for (int i = G.i0; i < G.i1; i++) {
            if (i + 2 <= G.i1) stage(G, i + 2, i + 2 < G.i1);   // reuses the slot of plane i-1
            cp_async_commit();
            cp_async_wait<1>();                 // planes i and i+1 have landed
            __syncthreads();
            const T* sb = smem + (size_t)slot_of(G, i) * STAGE;
            const T* sn = smem + (size_t)slot_of(G, i + 1) * STAGE;
            if (G.inside) {
                if constexpr (SPLIT) {
                    static_assert(CPT == 1, "split operands run one cell per thread");
                    const int col = IC + tx;
                    auto raw = [&](const T* b, int z, int row, int cc) { return b[z * ZT + row * W + cc]; };
                    const T a0 = raw(sb, 0, ty + 1, col), b0 = raw(sb, 1, ty + 1, col);
                    const T za[7] = {a0, zprev[0], raw(sn, 0, ty + 1, col), raw(sb, 0, ty, col), raw(sb, 0, ty + 2, col),
                                     raw(sb, 0, ty + 1, col - 1), raw(sb, 0, ty + 1, col + 1)};
                    const T zb[7] = {b0, zprev_b, raw(sn, 1, ty + 1, col), raw(sb, 1, ty, col), raw(sb, 1, ty + 2, col),
                                     raw(sb, 1, ty + 1, col - 1), raw(sb, 1, ty + 1, col + 1)};
                    T pv[NP];
#pragma unroll
                    for (int q = 0; q < NP; q++) pv[q] = sb[NZ * ZT + q * NCT + tid];
                    k.center2((int64_t)i * plane + G.o_own, za, zb, pv, acc);
                    zprev[0] = a0;
                    zprev_b = b0;
                } else if constexpr (CPT == 1) {
                    const int col = IC + tx;
                    const T zcur = zval(sb, ty + 1, col);
                    const T z7[7] = {zcur, zprev[0], zval(sn, ty + 1, col), zval(sb, ty, col), zval(sb, ty + 2, col),
                                     zval(sb, ty + 1, col - 1), zval(sb, ty + 1, col + 1)};
                    T pv[NP];
#pragma unroll
                    for (int q = 0; q < NP; q++) pv[q] = sb[NZ * ZT + q * NCT + tid];
                    k.center((int64_t)i * plane + G.o_own, z7, pv, acc);
                    zprev[0] = zcur;
                } else if constexpr (CPT == 2) {
                    // the thread's two cells as one 16-byte (8-byte for FP32)
                    // shared-memory load per row: consecutive threads read
                    // consecutive pairs, without bank conflicts
                    const int col = IC + 2 * tx;
                    auto zpair = [&](const T* b, int row, T& z0, T& z1) {
                        const Pair<T> a = ld_pair(b + row * W + col);
                        Pair<T> c2{T(0), T(0)};
                        if constexpr (NZ > 1) c2 = ld_pair(b + ZT + row * W + col);
                        z0 = k.zc(a.x, c2.x);
                        z1 = k.zc(a.y, c2.y);
                    };
                    T zc0, zc1, zn0, zn1, zs0, zs1, zt0, zt1;
                    zpair(sb, ty + 1, zc0, zc1);
                    zpair(sn, ty + 1, zn0, zn1);
                    zpair(sb, ty, zs0, zs1);
                    zpair(sb, ty + 2, zt0, zt1);
                    const T zw = zval(sb, ty + 1, col - 1), ze = zval(sb, ty + 1, col + 2);
                    T pv0[NP], pv1[NP];
#pragma unroll
                    for (int q = 0; q < NP; q++) {
                        const Pair<T> pq = ld_pair(sb + NZ * ZT + q * NCT + ty * TW + 2 * tx);
                        pv0[q] = pq.x;
                        pv1[q] = pq.y;
                    }
                    const T z70[7] = {zc0, zprev[0], zn0, zs0, zt0, zw, zc1};
                    k.center((int64_t)i * plane + G.o_own, z70, pv0, acc);
                    const T z71[7] = {zc1, zprev[1], zn1, zs1, zt1, zc0, ze};
                    k.center((int64_t)i * plane + G.o_own + 1, z71, pv1, acc);
                    zprev[0] = zc0;
                    zprev[1] = zc1;
                } else {
                    // four FP32 cells per thread: every row segment one 16-byte
                    // copy and one 16-byte shared-memory load
                    static_assert(CPT == 4 && sizeof(T) == 4, "four cells per thread: FP32");
                    const int col = IC + 4 * tx;
                    auto zquad = [&](const T* b, int row, T (&z)[4]) {
                        const float4 a = *reinterpret_cast<const float4*>(b + row * W + col);
                        float4 c2 = make_float4(0.f, 0.f, 0.f, 0.f);
                        if constexpr (NZ > 1) c2 = *reinterpret_cast<const float4*>(b + ZT + row * W + col);
                        z[0] = k.zc(a.x, c2.x);
                        z[1] = k.zc(a.y, c2.y);
                        z[2] = k.zc(a.z, c2.z);
                        z[3] = k.zc(a.w, c2.w);
                    };
                    T zc[4], zn[4], zs[4], zt[4];
                    zquad(sb, ty + 1, zc);
                    zquad(sn, ty + 1, zn);
                    zquad(sb, ty, zs);
                    zquad(sb, ty + 2, zt);
                    const T zw = zval(sb, ty + 1, col - 1), ze = zval(sb, ty + 1, col + 4);
                    T pv[4][NP];
#pragma unroll
                    for (int q = 0; q < NP; q++) {
                        const float4 pq = *reinterpret_cast<const float4*>(sb + NZ * ZT + q * NCT + ty * TW + 4 * tx);
                        pv[0][q] = pq.x;
                        pv[1][q] = pq.y;
                        pv[2][q] = pq.z;
                        pv[3][q] = pq.w;
                    }
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const T z7[7] = {zc[c], zprev[c], zn[c], zs[c], zt[c], c == 0 ? zw : zc[c - 1],
                                         c == 3 ? ze : zc[c + 1]};
                        k.center((int64_t)i * plane + G.o_own + c, z7, pv[c], acc);
                    }
#pragma unroll
                    for (int c = 0; c < 4; c++) zprev[c] = zc[c];
                }
            }
            __syncthreads();                    // slot of plane i is free for plane i+3
        }
        cp_async_wait<0>();
        const int next = s_next;                // written before this item's barriers
        Geo GN = G;
        if (next < m.nitems) {
            GN = geometry(next);
            prologue(GN);                       // every plane of this item has been read
        }
        if constexpr (K::Q > 0) {
            double tot[K::Q];
            if (item_reduce<K::Q>(acc, partials, m.item_base + item, m.nitems_total ? m.nitems_total : m.nitems,
                                  &st->count, tot) &&
                tid == 0)
                k.done(st, tot);
        }
        __syncthreads();                        // s_next is rewritten at the next item's start
        item = next;
        G = GN;
    }
    cp_async_wait<0>();
    // the last block out resets the queue for the next launch
    if (tid == 0) {
        const unsigned prev = atomicAdd(&st->exitc, 1u);
        if (prev == gridDim.x - 1) {
            st->queue = 0u;
            st->exitc = 0u;
            __threadfence();
        }
    }
}

template <class K, int CPT, bool HALO, bool PAIR>
inline int launch_march_k(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const K& kern, SolverState* st,
                          double* partials) {
    const int ic = PAIR ? 16 / (int)sizeof(typename K::type) : m.cpt;   // first interior column of an operand row
    const size_t smem = 3 * march_stage_elems<K>(m.block.x * m.cpt, m.block.y, ic) * sizeof(typename K::type);
    static int per_sm = 0;
    static size_t per_sm_smem = 0;
    if (per_sm == 0 || per_sm_smem != smem) {
        if (smem > 48 * 1024)
            DARE_CUDA(ctx, cudaFuncSetAttribute(k_march<K, CPT, HALO, PAIR>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_march<K, CPT, HALO, PAIR>, m.block.x * m.block.y,
                                                      smem);
        if (per_sm < 1) per_sm = 1;
        per_sm_smem = smem;
    }
    int blocks = per_sm * ctx->num_sms;
    if (blocks > m.nitems) blocks = m.nitems;
    k_march<K, CPT, HALO, PAIR><<<blocks, m.block, smem, ctx->stream>>>(g, kern, st, partials, m);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// 16-byte staging (one copy = 16 / sizeof(T) cells): a row length and tile
// width that are multiples of it, enough threads for the operand copies, and
// 16-byte aligned arrays
template <class K, bool HALO>
inline bool march_pairs_ok(const GridDev& g, const MarchCfg& m, const K& kern, int cpt) {
    const int vec = 16 / (int)sizeof(typename K::type);
    const int nt = (int)(m.block.x * m.block.y), tw = (int)m.block.x * cpt, tj = (int)m.block.y;
    bool ok = g.n[2] % vec == 0 && tw % vec == 0 && (tj + 2) * (tw / vec) + 2 * tj <= nt;
    for (int q = 0; q < K::NP; q++) ok = ok && ((uintptr_t)kern.ps[q] & 15) == 0;
    for (int z = 0; z < K::NZ; z++) {
        ok = ok && ((uintptr_t)kern.zs[z] & 15) == 0;
        if (HALO)
            for (int h = 0; h < 2; h++) ok = ok && ((uintptr_t)m.halo[z][h] & 15) == 0;
    }
    return ok;
}

template <class K, int CPT, bool HALO>
inline int launch_march_t(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const K& kern, SolverState* st,
                          double* partials) {
    if constexpr ((CPT == 1 && sizeof(typename K::type) == 8) || (CPT == 2 && sizeof(typename K::type) == 4)) {
        if (march_pairs_ok<K, HALO>(g, m, kern, CPT))
            return launch_march_k<K, CPT, HALO, true>(ctx, g, m, kern, st, partials);
    }
    return launch_march_k<K, CPT, HALO, false>(ctx, g, m, kern, st, partials);
}

// Two cells per thread (K::kPairs) paid off for steps 1, 2 and 3 while one
// cell per thread staged every value with its own 8-byte copy (256^3: 0.291
// -> 0.257 ms for step 1).  With the 16-byte paired staging of the FP64
// one-cell kernels (PAIR in k_march) one cell per thread is ahead again
// (step 1 0.255 -> 0.252 ms, step 2 0.254 -> 0.249, step 3 0.252 -> 0.249),
// so the FP64 steps run one cell per thread on 32 x 8 tiles; the FP32
// kernels keep two or four cells per thread.  With eight streams and five
// dot products (step 4: 0.316 -> 0.404 ms with two cells), or many outputs
// per cell (init: 0.29 -> 0.38 ms, fold), two cells per thread never paid.
// HALO: the slab variant, which reads m.halo (ignored otherwise).
template <class K, bool HALO = false>
inline int launch_march(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const K& kern, SolverState* st,
                        double* partials) {
    if (m.nitems > kMaxBlocks || m.item_base + m.nitems > kMaxBlocks || m.nitems_total > kMaxBlocks)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "grid too large for the reduction");
    if (m.cpt == 4) {   // FP32 grids with n2 a multiple of 4, 64-cell tiles
        if constexpr (sizeof(typename K::type) == 4 && !SplitOperands<K>::value) {
            MarchCfg m2 = m;   // two cells per thread on the same tiles, 16-byte staging
            m2.cpt = 2;
            m2.block = dim3(m.block.x * 2, m.block.y, 1);
            if (march_pairs_ok<K, HALO>(g, m2, kern, 2)) return launch_march_k<K, 2, HALO, true>(ctx, g, m2, kern, st, partials);
            if constexpr (K::kPairs) {
                return launch_march_t<K, 4, HALO>(ctx, g, m, kern, st, partials);
            } else {
                MarchCfg m2 = m;   // two cells per thread on the same tiles
                m2.cpt = 2;
                m2.block = dim3(m.block.x * 2, m.block.y, 1);
                return launch_march_t<K, 2, HALO>(ctx, g, m2, kern, st, partials);
            }
        }
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "four cells per thread are for FP32 kernels");
    }
    if constexpr (K::kPairs) {
        if (m.cpt == 2) return launch_march_t<K, 2, HALO>(ctx, g, m, kern, st, partials);
    }
    if (m.cpt == 1) return launch_march_t<K, 1, HALO>(ctx, g, m, kern, st, partials);
    MarchCfg m1 = m;   // the same tiles, one cell per thread
    m1.cpt = 1;
    m1.block = dim3(m.block.x * m.cpt, m.block.y, 1);
    return launch_march_t<K, 1, HALO>(ctx, g, m1, kern, st, partials);
}

// K5: the deferred steps (10) x = x + alpha1 u1 and (15) u = r1 - beta u1
//     (u1 the u of step (5), r1 the r of step (8)), then (24)
//     x = x + w1 r + w2 s + alpha u; (25) r = r - w1 s - w2 t; ||r||;
//     u = u - w1 v - w2 w; then the next iteration's (3), (4).
//     `base` / `total`: partial-sum slots shared with other launches (slabs;
//     0, 0: this launch alone).  `vec4` (FP32 only; n % 4 == 0 and every
//     array 16-byte aligned): four cells per thread and 16-byte accesses
//     (512^3: 0.92 ms; with 4-byte accesses the FP32 kernel took 1.22 ms,
//     81 % of copy bandwidth).
template <typename T>
__global__ void __launch_bounds__(256) k_step5(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                               const T* __restrict__ s, const T* __restrict__ t,
                                               T* __restrict__ u, const T* __restrict__ u1,
                                               const T* __restrict__ r1, const T* __restrict__ v,
                                               const T* __restrict__ w, const T* __restrict__ rh, SolverState* st,
                                               double* partials, int base, int total, int vec4) {
    if (st->done) return;
    const T w1 = (T)st->omega1, w2 = (T)st->omega2, alpha = (T)st->alpha, alpha1 = (T)st->alpha1;
    const T beta = (T)st->beta;
    double acc[2] = {0., 0.};
    if constexpr (sizeof(T) == 4) {
        if (vec4) {
            // the scalar loop's expressions, cell by cell within each float4
            auto cell = [&](float rc, float sc, float u1c, float xc0, float r1c, float tc, float vc, float wc,
                            float rhc, float& xo, float& ro, float& uo) {
                const float x10 = alpha1 * u1c + xc0;
                const float u15 = r1c - beta * u1c;
                float xc = w1 * rc + w2 * sc + x10;
                xc = alpha * u15 + xc;
                xo = xc;
                const float rn = -w1 * sc + -w2 * tc + rc;
                ro = rn;
                uo = -w1 * vc + -w2 * wc + u15;
                acc[0] += (double)rn * (double)rn;
                acc[1] += (double)rhc * (double)rn;
            };
            const int64_t n4 = n >> 2;
            for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n4;
                 q += (int64_t)gridDim.x * blockDim.x) {
                const float4 rq = reinterpret_cast<const float4*>(r)[q], sq = reinterpret_cast<const float4*>(s)[q];
                const float4 u1q = reinterpret_cast<const float4*>(u1)[q], xq = reinterpret_cast<const float4*>(x)[q];
                const float4 r1q = reinterpret_cast<const float4*>(r1)[q], tq = reinterpret_cast<const float4*>(t)[q];
                const float4 vq = reinterpret_cast<const float4*>(v)[q], wq = reinterpret_cast<const float4*>(w)[q];
                const float4 rhq = reinterpret_cast<const float4*>(rh)[q];
                float4 xo, ro, uo;
                cell(rq.x, sq.x, u1q.x, xq.x, r1q.x, tq.x, vq.x, wq.x, rhq.x, xo.x, ro.x, uo.x);
                cell(rq.y, sq.y, u1q.y, xq.y, r1q.y, tq.y, vq.y, wq.y, rhq.y, xo.y, ro.y, uo.y);
                cell(rq.z, sq.z, u1q.z, xq.z, r1q.z, tq.z, vq.z, wq.z, rhq.z, xo.z, ro.z, uo.z);
                cell(rq.w, sq.w, u1q.w, xq.w, r1q.w, tq.w, vq.w, wq.w, rhq.w, xo.w, ro.w, uo.w);
                reinterpret_cast<float4*>(x)[q] = xo;
                reinterpret_cast<float4*>(r)[q] = ro;
                reinterpret_cast<float4*>(u)[q] = uo;
            }
            n = 0;   // the scalar loop below has nothing left to do
        }
    }
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const T rc = r[c], sc = s[c], u1c = u1[c];
        const T x10 = alpha1 * u1c + x[c];
        const T u15 = r1[c] - beta * u1c;
        T xc = w1 * rc + w2 * sc + x10;
        xc = alpha * u15 + xc;
        x[c] = xc;
        const T rn = -w1 * sc + -w2 * t[c] + rc;
        r[c] = rn;
        u[c] = -w1 * v[c] + -w2 * w[c] + u15;
        acc[0] += (double)rn * (double)rn;
        acc[1] += (double)rh[c] * (double)rn;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &st->count, tot, base, total)) return;
    if (threadIdx.x == 0) finish_update(st, tot);
}

// Step (10) of an iteration that stopped after it and before K5 (a
// breakdown in steps (14), (20) or (21)): x = x + alpha1 u1.
inline __host__ __device__ bool step10_pending_state(int status, int step) {
    return status == ST_TAU0 || (status == ST_BREAKDOWN && (step == 14 || step == 20));
}
template <typename T>
__global__ void k_step10(int64_t n, const SolverState* st, const T* __restrict__ u1, T* __restrict__ x) {
    if (!step10_pending_state(st->status, st->step)) return;   // read on the device: no host round trip
    const T alpha1 = (T)st->alpha1;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        x[c] = alpha1 * u1[c] + x[c];
}
inline bool step10_pending(const SolverState& st) { return step10_pending_state(st.status, st.step); }


static __global__ void k_invdiag(const double* __restrict__ dc, double* __restrict__ invd, int64_t n) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        invd[c] = 1. / dc[c];
}

// x = invd .* x (applyRightPrec at the end of the solve)
static __global__ void k_scale(int64_t n, const double* __restrict__ invd, double* __restrict__ x) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        x[c] = invd[c] * x[c];
}

}  // namespace dare_gpu
