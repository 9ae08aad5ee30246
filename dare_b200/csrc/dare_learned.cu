// dare_learned.cu -- BiCGStab2 with the learned linear preconditioner,
// FP32 inside an FP64 iterative refinement, with the automatic fallback to
// the plain FP64 Jacobi-BiCGStab2.
//
//   outer (FP64):  r = b - A x; stop when ||r||_2 <= tol_abs
//   inner (FP32):  BiCGStab(2) on  Ahat N y = r,  Ahat = A D^-1 (unit
//                  diagonal), N the U-Net, from zero, FP64 dot products and
//                  scalar recurrences (the reference's steps 3-25,
//                  BiCGStab2.inl:262-560, with the operator Ahat N), in
//                  flexible form (below)
//   update (FP64): x += D^-1 d,  d the inner solution in the x variable
//
// Flexible form.  The network is linear in exact arithmetic but its BF16
// activations make N(a + b) differ from N(a) + N(b) by a few 1e-3, so the
// textbook right-preconditioned update (accumulate y, apply N once at the
// end) would leave the recurrence residual inconsistent with the iterate at
// that level.  Instead every iteration keeps the four network outputs it
// computes, zu = N(u) (step 6), zr = N(r) (step 9), zv = N(v) (step 13),
// zs = N(s) (step 18), and updates the x-variable correction directly,
//     d += (a1 - a2 b1) zu + (a2 + w1) zr - w1 a2 zv + w2 zs,
// the x-space image of the reference's y updates (steps 10 and 24) written
// with exactly the vectors whose Ahat-images (v, s, w, t) entered the
// residual recurrence (steps 8, 16, 25).  The recurrence residual is then
// the residual of d up to FP32 rounding, however nonlinear N is.
// The learned phase stops when its inner iterations exceed the iteration
// budget or the refinement stops contracting; the plain FP64 solve then
// continues from the current iterate.  The reported residual is always the
// FP64 ||b - A x||_2.
//
// One inner iteration is one CUDA graph: 4 network applications (13
// tensor-core/level-transfer kernels each), 4 SpMV kernels with fused dot
// products (plane-marching, dare_march.cuh), 6 vector kernels.  The FP64
// residual of the refinement also runs in the marching engine and is read
// back with the inner solve's state.
// The inner solve may stop after its first iteration (the reference's
// `k > 1` rule applies to its own solve, not to this inner correction).
// Scalars live on the device; kernels after a breakdown see `done` and skip
// their work.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "dare_march.cuh"
#include "dare_unet.cuh"

using namespace dare_gpu;

namespace dare_gpu {
namespace learned {

// The solve's scalars live in a SolverState (the marching kernels' queue
// and reduction counters are part of it); status codes ST_*.
struct Vecs {
    float *rh, *r, *u, *v, *s, *w, *t, *d, *zu, *zr, *zv, *zs, *rin;
};
constexpr int kNumVecs = 13;

}  // namespace learned
}  // namespace dare_gpu

struct dare_learned_ws {
    int64_t n = 0;
    float* ahat32 = nullptr;   // 6 n
    float* vec = nullptr;      // kNumVecs n
    double* partials = nullptr;
    double* scal = nullptr;    // [0] outer norms
    dare_gpu::SolverState* st = nullptr;
    dare_gpu::SolverState* st_host = nullptr;
    dare_gpu::MarchCfg march32;   // tiles of the FP32 marching kernels
    cudaGraphExec_t graph = nullptr;
    const dare_unet* graph_net = nullptr;
    int64_t graph_kernels = 0;  // kernels in one captured iteration
};

void dare_learned_ws_free(dare_learned_ws* lw) {
    if (!lw) return;
    if (lw->graph) cudaGraphExecDestroy(lw->graph);
    cudaFree(lw->ahat32);
    cudaFree(lw->vec);
    cudaFree(lw->partials);
    cudaFree(lw->scal);
    cudaFree(lw->st);
    if (lw->st_host) cudaFreeHost(lw->st_host);
    delete lw;
}

namespace dare_gpu {
namespace learned {

#define GRID_LOOP(c, n) \
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < (n); c += (int64_t)gridDim.x * blockDim.x)

// r = b - A x with the assembled FP64 operator, stored as FP32 for the inner
// solve, and ||r||_2 -> *out
struct FLResidual {
    using type = double;
    static constexpr int Q = 1, NZ = 1, NP = 8;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;
    const double* zs[2];   // x
    const double* ps[NP];  // 7 coefficients, b
    float* rin;
    double* out;
    __device__ void load(const SolverState*) {}
    __device__ double zc(double a, double) const { return a; }
    __device__ void center(int64_t c, const double (&zz)[7], const double* p, double* acc) const {
        const double r = p[7] - apply_pre<double, false>(p, zz);
        rin[c] = (float)r;
        acc[0] += r * r;
    }
    __device__ void done(SolverState*, const double* tot) const { *out = sqrt(tot[0]); }
};

__device__ __forceinline__ void fail(SolverState* st, int step) {
    st->done = 1;
    st->status = ST_BREAKDOWN;
    st->step = step;
}

// out = Ahat z for a network output z, with <out, r_hat_0>.  MODE 0 (steps
// 6-7 and 13-14): gamma -> alpha = rho0 / gamma; MODE 1 (steps 9-11):
// rho1 -> beta = alpha rho1 / rho0.
template <int MODE, int STEP>
struct FLSpmvDot {
    using type = float;
    static constexpr int Q = 1, NZ = 1, NC = 6, NP = 7;
    static constexpr bool kCheckDone = true;
    static constexpr bool kPairs = true;   // two cells per thread (see launch_march)
    const float* zs[2];   // z
    const float* ps[NP];  // 6 folded off-diagonals, r_hat_0
    float* out;
    __device__ void load(const SolverState*) {}
    __device__ float zc(float a, float) const { return a; }
    __device__ void center(int64_t c, const float (&zz)[7], const float* p, double* acc) const {
        const float v = apply_pre<float, true>(p, zz);
        out[c] = v;
        acc[0] += (double)v * (double)p[NC];
    }
    __device__ void done(SolverState* st, const double* tot) const {
        if (MODE == 0) {
            if (tot[0] == 0.) return fail(st, STEP);
            st->alpha = st->rho0 / tot[0];
            if (STEP == 7) st->alpha1 = st->alpha;
        } else {
            st->beta = st->alpha * tot[0] / st->rho0;
            st->beta1 = st->beta;
            st->rho0 = tot[0];
        }
    }
};

// (18)-(23): t = Ahat zs; <r,s>, <s,s>, <s,t>, <t,t>, <r,t>; omega1, omega2
struct FLSpmvOmega {
    using type = float;
    static constexpr int Q = 5, NZ = 1, NC = 6, NP = 8;
    static constexpr bool kCheckDone = true;
    static constexpr bool kPairs = false;
    const float* zs[2];   // zs
    const float* ps[NP];  // 6 folded off-diagonals, r, s
    float* t;
    __device__ void load(const SolverState*) {}
    __device__ float zc(float a, float) const { return a; }
    __device__ void center(int64_t c, const float (&zz)[7], const float* p, double* acc) const {
        const float tv = apply_pre<float, true>(p, zz);
        t[c] = tv;
        const double r = p[NC], s = p[NC + 1], td = tv;
        acc[0] += r * s;
        acc[1] += s * s;
        acc[2] += s * td;
        acc[3] += td * td;
        acc[4] += r * td;
    }
    __device__ void done(SolverState* st, const double* tot) const {
        double om1 = tot[0], mu = tot[1], nu = tot[2], tau = tot[3], om2 = tot[4];
        if (mu == 0.) return fail(st, 20);
        tau -= nu * nu / mu;
        if (tau == 0.) return fail(st, 21);
        om2 = (om2 - nu * om1 / mu) / tau;
        om1 = (om1 - nu * om2) / mu;
        st->omega1 = om1;
        st->omega2 = om2;
    }
};

__global__ void __launch_bounds__(256) k_bnorm(int64_t n, const double* __restrict__ b, SolverState* st, double* partials,
                                               double* out) {
    double acc[1] = {0.};
    GRID_LOOP(c, n) acc[0] += b[c] * b[c];
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) *out = sqrt(tot[0]);
}

// The vector kernels below work on four cells at a time (16-byte accesses):
// the learned solve's grids have sizes that are multiples of 8, so n is a
// multiple of 4 and every vector of the workspace starts 16-byte aligned.
__device__ __forceinline__ float4 ld4(const float* p, int64_t q) { return reinterpret_cast<const float4*>(p)[q]; }
__device__ __forceinline__ void st4(float* p, int64_t q, float4 v) { reinterpret_cast<float4*>(p)[q] = v; }
__device__ __forceinline__ double sq4(float4 a) {
    return (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z + (double)a.w * a.w;
}
__device__ __forceinline__ double dot4(float4 a, float4 b) {
    return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
}
// a - c b, component by component
__device__ __forceinline__ float4 axmy(float4 a, float c, float4 b) {
    return make_float4(a.x - c * b.x, a.y - c * b.y, a.z - c * b.z, a.w - c * b.w);
}

// start of an inner solve: r = rh = rin, u = v = w = d = 0
__global__ void __launch_bounds__(256) k_init(int64_t n, Vecs vs, SolverState* st, double* partials, double rel_tol,
                                              int max_it) {
    double acc[1] = {0.};
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    GRID_LOOP(q, n / 4) {
        const float4 r = ld4(vs.rin, q);
        st4(vs.r, q, r);
        st4(vs.rh, q, r);
        st4(vs.u, q, zero);
        st4(vs.v, q, zero);
        st4(vs.w, q, zero);
        st4(vs.d, q, zero);
        acc[0] += sq4(r);
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        st->rnorm0 = sqrt(tot[0]);
        st->rnorm = st->rnorm0;
        st->tol = rel_tol * st->rnorm0;
        st->rho0 = st->omega1 = st->omega2 = 1.;
        st->alpha = 0.;
        st->beta = 0.;
        st->k = 1;
        st->max_it = max_it;
        st->status = ST_RUNNING;
        st->step = 0;
        st->done = (st->rnorm0 == 0.) ? 1 : 0;
        if (st->done) st->status = ST_CONVERGED;
        if (!(st->rnorm0 == st->rnorm0)) {
            st->done = 1;
            st->status = ST_NAN;
        }
    }
}

// (3), (4): rho1 = <rh, r>, beta
__global__ void __launch_bounds__(256) k_rho(int64_t n, Vecs vs, SolverState* st, double* partials) {
    if (st->done) return;
    double acc[1] = {0.};
    GRID_LOOP(q, n / 4) acc[0] += dot4(ld4(vs.rh, q), ld4(vs.r, q));
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        st->rho0 = -st->omega2 * st->rho0;
        if (st->rho0 == 0.) return fail(st, 3);
        const double rho1 = tot[0];
        st->beta = st->alpha * rho1 / st->rho0;
        st->rho0 = rho1;
        if (st->rho0 == 0.) return fail(st, 4);
    }
}

// (5) u = r - beta u
__global__ void k_upd_u(int64_t n, Vecs vs, const SolverState* st) {
    if (st->done) return;
    const float beta = (float)st->beta;
    GRID_LOOP(q, n / 4) st4(vs.u, q, axmy(ld4(vs.r, q), beta, ld4(vs.u, q)));
}

// (8): r -= alpha v (the matching x update is folded into k_upd_final)
__global__ void k_upd_r(int64_t n, Vecs vs, const SolverState* st) {
    if (st->done) return;
    const float alpha = (float)st->alpha;
    GRID_LOOP(q, n / 4) st4(vs.r, q, axmy(ld4(vs.r, q), alpha, ld4(vs.v, q)));
}

// (12) v = s - beta v
__global__ void k_upd_v(int64_t n, Vecs vs, const SolverState* st) {
    if (st->done) return;
    const float beta = (float)st->beta;
    GRID_LOOP(q, n / 4) st4(vs.v, q, axmy(ld4(vs.s, q), beta, ld4(vs.v, q)));
}

// (15)-(17)
__global__ void k_upd3(int64_t n, Vecs vs, const SolverState* st) {
    if (st->done) return;
    const float alpha = (float)st->alpha, beta = (float)st->beta;
    GRID_LOOP(q, n / 4) {
        const float4 r = ld4(vs.r, q);
        st4(vs.u, q, axmy(r, beta, ld4(vs.u, q)));
        st4(vs.r, q, axmy(r, alpha, ld4(vs.v, q)));
        st4(vs.s, q, axmy(ld4(vs.s, q), alpha, ld4(vs.w, q)));
    }
}

// (10), (24) in flexible form: d += (a1 - a2 b1) zu + (a2 + w1) zr - w1 a2 zv + w2 zs;
// (25): r -= w1 s + w2 t; u -= w1 v + w2 w; convergence test on ||r||
__global__ void __launch_bounds__(256) k_upd_final(int64_t n, Vecs vs, SolverState* st, double* partials) {
    if (st->done) return;
    const double a1 = st->alpha1, a2 = st->alpha, b1 = st->beta1, om1 = st->omega1, om2 = st->omega2;
    const float cu = (float)(a1 - a2 * b1), cr = (float)(a2 + om1), cv = (float)(-om1 * a2), cs = (float)om2;
    const float w1 = (float)om1, w2 = (float)om2;
    double acc[1] = {0.};
    GRID_LOOP(q, n / 4) {
        const float4 zu = ld4(vs.zu, q), zr = ld4(vs.zr, q), zv = ld4(vs.zv, q), zs = ld4(vs.zs, q);
        float4 d = ld4(vs.d, q);
        d.x += cu * zu.x + cr * zr.x + cv * zv.x + cs * zs.x;
        d.y += cu * zu.y + cr * zr.y + cv * zv.y + cs * zs.y;
        d.z += cu * zu.z + cr * zr.z + cv * zv.z + cs * zs.z;
        d.w += cu * zu.w + cr * zr.w + cv * zv.w + cs * zs.w;
        st4(vs.d, q, d);
        const float4 r = ld4(vs.r, q), s = ld4(vs.s, q), t = ld4(vs.t, q);
        const float4 rn = make_float4(r.x - w1 * s.x - w2 * t.x, r.y - w1 * s.y - w2 * t.y,
                                      r.z - w1 * s.z - w2 * t.z, r.w - w1 * s.w - w2 * t.w);
        st4(vs.r, q, rn);
        const float4 v = ld4(vs.v, q), w = ld4(vs.w, q);
        float4 u = ld4(vs.u, q);
        u.x -= w1 * v.x + w2 * w.x;
        u.y -= w1 * v.y + w2 * w.y;
        u.z -= w1 * v.z + w2 * w.z;
        u.w -= w1 * v.w + w2 * w.w;
        st4(vs.u, q, u);
        acc[0] += sq4(rn);
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        const double rn = sqrt(tot[0]);
        st->rnorm = rn;
        if (!(rn == rn)) {
            st->done = 1;
            st->status = ST_NAN;
        } else if (rn <= st->tol) {
            st->done = 1;
            st->status = ST_CONVERGED;
        } else if (++st->k > st->max_it) {
            st->done = 1;
            st->status = ST_MAXIT;
        }
    }
}

// x += D^-1 z (FP64), unless the inner solve ended in NaN (read on the device)
__global__ void k_correct(int64_t n, const double* __restrict__ invd, const float* __restrict__ z,
                          double* __restrict__ x, const SolverState* st) {
    if (st->status == ST_NAN) return;
    GRID_LOOP(c, n) x[c] += invd[c] * (double)z[c];
}


__global__ void k_to_precond_var(int64_t n, const double* __restrict__ dc, double* __restrict__ x) {
    GRID_LOOP(c, n) x[c] = dc[c] * x[c];
}

static int launch_iteration(dare_ctx* ctx, dare_unet* net, const GridDev& g, const MarchCfg& m, const float* ah,
                            const Vecs& vs, SolverState* st, double* partials) {
    const int64_t n = g.ncell;
    const int eb = grid_blocks(ctx, n, 256, 8);
    cudaStream_t s = ctx->stream;
    int rc;
    auto spmv_dot = [&](auto f, const float* z, float* out) {
        f.zs[0] = z;
        for (int q = 0; q < 6; q++) f.ps[q] = ah + (size_t)q * n;
        f.ps[6] = vs.rh;
        f.out = out;
        return launch_march(ctx, g, m, f, st, partials);
    };
    k_rho<<<eb, 256, 0, s>>>(n, vs, st, partials);
    DARE_LAUNCHED(ctx);
    k_upd_u<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.u, vs.zu))) return rc;
    if ((rc = spmv_dot(FLSpmvDot<0, 7>{}, vs.zu, vs.v))) return rc;
    k_upd_r<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.r, vs.zr))) return rc;
    if ((rc = spmv_dot(FLSpmvDot<1, 11>{}, vs.zr, vs.s))) return rc;
    k_upd_v<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.v, vs.zv))) return rc;
    if ((rc = spmv_dot(FLSpmvDot<0, 14>{}, vs.zv, vs.w))) return rc;
    k_upd3<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.s, vs.zs))) return rc;
    FLSpmvOmega fo{};
    fo.zs[0] = vs.zs;
    for (int q = 0; q < 6; q++) fo.ps[q] = ah + (size_t)q * n;
    fo.ps[6] = vs.r;
    fo.ps[7] = vs.s;
    fo.t = vs.t;
    if ((rc = launch_march(ctx, g, m, fo, st, partials))) return rc;
    k_upd_final<<<eb, 256, 0, s>>>(n, vs, st, partials);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

static int read_scalar(dare_ctx* ctx, const double* d, double* h) {
    DARE_CUDA(ctx, cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

}  // namespace learned
}  // namespace dare_gpu

extern "C" void dare_learned_params_default(dare_learned_params* p) {
    if (!p) return;
    p->iteration_budget = 40;
    p->inner_max_it = 20;
    p->inner_rel_tol = 1e-4;
    p->max_refinements = 12;
}

extern "C" int dare_bicgstab2_learned(dare_system* s, dare_unet* net, const dare_solver_params* p,
                                      const dare_learned_params* lp, dare_solve_report* rep) {
    using namespace dare_gpu::learned;
    if (!s || !net || !p || !lp || !rep) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->grid->dev;
    if (net->ctx != ctx) return set_error(ctx, DARE_ERR_BAD_ARG, "bicgstab2_learned: network on another context");
    if (s->ncomp != 1)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "bicgstab2_learned: the network preconditions one field component");
    const int* sys_n = net->coarse ? net->fine : net->n;
    if (g.dim != 3 || g.n[0] != sys_n[0] || g.n[1] != sys_n[1] || g.n[2] != sys_n[2])
        return set_error(ctx, DARE_ERR_BAD_ARG, "bicgstab2_learned: grid does not match the network");
    if (g.ncell % 4)   // the vector kernels take four cells at a time (sizes are multiples of 8)
        return set_error(ctx, DARE_ERR_BAD_ARG, "bicgstab2_learned: cell count must be a multiple of 4");
    if (lp->iteration_budget < 1 || lp->inner_max_it < 1 || !(lp->inner_rel_tol > 0.))
        return set_error(ctx, DARE_ERR_BAD_ARG, "bicgstab2_learned: bad learned parameters");
    cudaSetDevice(ctx->device);
    int rc = ensure_solver_ws(s);
    if (rc) return rc;
    dare_solver_ws* ws = s->ws;
    const int64_t n = g.ncell;
    if (!ws->learned) {
        dare_learned_ws* lw = new (std::nothrow) dare_learned_ws();
        if (!lw) return DARE_ERR_OOM;
        lw->n = n;
        cudaError_t e = cudaMalloc(&lw->ahat32, (size_t)n * 6 * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&lw->vec, (size_t)n * kNumVecs * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&lw->partials, (size_t)kMaxQ * kMaxBlocks * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&lw->scal, 4 * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&lw->st, sizeof(SolverState));
        if (e == cudaSuccess) e = cudaMemset(lw->st, 0, sizeof(SolverState));
        if (e == cudaSuccess) e = cudaMallocHost(&lw->st_host, sizeof(SolverState));
        if (e != cudaSuccess) {
            dare_learned_ws_free(lw);
            return check_cuda(ctx, e, "bicgstab2_learned workspace");
        }
        lw->march32 = march_config(ctx, g, sizeof(float));
        ws->learned = lw;
    }
    dare_learned_ws* lw = ws->learned;
    const int eb = grid_blocks(ctx, n, 256, 8);
    float* V = lw->vec;
    Vecs vs;
    float** slots[kNumVecs] = {&vs.rh, &vs.r, &vs.u, &vs.v, &vs.s, &vs.w, &vs.t,
                               &vs.d, &vs.zu, &vs.zr, &vs.zv, &vs.zs, &vs.rin};
    for (int i = 0; i < kNumVecs; i++) *slots[i] = V + (size_t)i * n;

    // Ahat = A D^-1, folded straight to FP32
    if ((rc = launch_fold32(ctx, g, ws->march, s->diag, ws->invd, lw->ahat32, ws->st, ws->partials))) return rc;
    DARE_CUDA(ctx, cudaMemsetAsync(lw->st, 0, sizeof(SolverState), ctx->stream));
    k_bnorm<<<eb, 256, 0, ctx->stream>>>(n, s->rhs, lw->st, lw->partials, lw->scal);
    DARE_LAUNCHED(ctx);
    double bnorm = 0.;
    if ((rc = read_scalar(ctx, lw->scal, &bnorm))) return rc;
    const double tol_abs = p->tol_relative ? p->tol * bnorm : p->tol;

    // one CUDA graph per inner iteration (captured once per network and
    // system); the host replays it and polls the state
    if (!lw->graph || lw->graph_net != net) {
        if (lw->graph) cudaGraphExecDestroy(lw->graph);
        lw->graph = nullptr;
        if ((rc = dare_gpu::unet::apply(net, vs.rin, vs.zs))) return rc;  // sets the launch configurations
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaGraph_t graph = nullptr;
        DARE_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = ctx->launches;
        rc = launch_iteration(ctx, net, g, lw->march32, lw->ahat32, vs, lw->st, lw->partials);
        lw->graph_kernels = ctx->launches - before;
        ctx->launches = before;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return check_cuda(ctx, e, "bicgstab2_learned capture");
        e = cudaGraphInstantiate(&lw->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return check_cuda(ctx, e, "bicgstab2_learned instantiate");
        lw->graph_net = net;
    }

    std::memset(rep, 0, sizeof(*rep));
    rep->b_norm = bnorm;
    rep->tol_abs = tol_abs;
    double rnorm = 0., prev = INFINITY;
    bool converged = false;
    int refinements = 0, inner_total = 0;
    // r = b - A x into the inner right-hand side, its norm into out
    auto residual = [&](double* out) {
        FLResidual fr{};
        fr.zs[0] = s->x;
        set_coef_streams<double, false, 8>(OpT<double>{s->diag, s->diag + n, n}, fr.ps);   // W..T, then C
        fr.ps[7] = s->rhs;
        fr.rin = vs.rin;
        fr.out = out;
        return launch_march(ctx, g, ws->march, fr, lw->st, lw->partials);
    };
    if ((rc = residual(lw->scal))) return rc;
    if ((rc = read_scalar(ctx, lw->scal, &rnorm))) return rc;
    for (int it = 0;; it++) {
        if (rnorm <= tol_abs) {
            converged = true;
            break;
        }
        if (!(rnorm < 0.5 * prev) || it >= lp->max_refinements || inner_total >= lp->iteration_budget) break;
        prev = rnorm;
        const int cap = std::min(lp->inner_max_it, lp->iteration_budget - inner_total);
        k_init<<<eb, 256, 0, ctx->stream>>>(n, vs, lw->st, lw->partials, lp->inner_rel_tol, cap);
        DARE_LAUNCHED(ctx);
        for (int j = 0; j < cap; j++) {
            DARE_CUDA(ctx, cudaGraphLaunch(lw->graph, ctx->stream));
            ctx->launches += lw->graph_kernels;
            DARE_CUDA(ctx, cudaMemcpyAsync(lw->st_host, lw->st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx->stream));
            DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (lw->st_host->done) break;
        }
        // x += D^-1 d (skipped on the device after a NaN) and the next
        // residual, read back with the inner solve's state in one round trip
        k_correct<<<eb, 256, 0, ctx->stream>>>(n, ws->invd, vs.d, s->x, lw->st);
        DARE_LAUNCHED(ctx);
        if ((rc = residual(&lw->st->tres))) return rc;
        DARE_CUDA(ctx, cudaMemcpyAsync(lw->st_host, lw->st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        const SolverState st = *lw->st_host;
        inner_total += std::min(st.k, cap);
        if (st.status == ST_NAN) break;
        rnorm = st.tres;
        refinements++;
    }
    rep->refinements = refinements;
    rep->inner_iters = inner_total;
    rep->iters = inner_total;
    rep->res_abs = rnorm;
    rep->true_res_abs = rnorm;
    if (converged) {
        rep->converged = 1;
        rep->status = DARE_SOLVE_CONVERGED;
        return DARE_OK;
    }
    // the plain FP64 Jacobi-BiCGStab2 from the current iterate (its variable is y = D x)
    k_to_precond_var<<<eb, 256, 0, ctx->stream>>>(n, s->diag, s->x);
    DARE_LAUNCHED(ctx);
    dare_solver_params q = *p;
    q.precond = DARE_PREC_JACOBI;
    q.precision = DARE_PRECISION_FP64;
    q.tol = tol_abs;
    q.tol_relative = 0;
    q.compute_true_residual = 1;
    dare_solve_report r2;
    if ((rc = dare_bicgstab2_fp64(s, &q, &r2))) return rc;
    *rep = r2;
    rep->iters = inner_total + r2.iters;
    rep->refinements = refinements;
    rep->inner_iters = inner_total;
    rep->fallback_used = 1;
    rep->b_norm = bnorm;
    rep->tol_abs = tol_abs;
    return DARE_OK;
}
