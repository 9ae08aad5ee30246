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
// One inner iteration is one CUDA graph: 4 network applications (11
// tensor-core/level-transfer kernels each), 4 SpMV kernels with fused dot
// products, 5 vector kernels.  The inner solve may stop after its first
// iteration (the reference's `k > 1` rule applies to its own solve, not to
// this inner correction).  Scalars live on the device; kernels after a
// breakdown see `done` and skip their work.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "dare_bicgstab2.cuh"
#include "dare_unet.cuh"

using namespace dare_gpu;

namespace dare_gpu {
namespace learned {

enum : int { L_RUNNING = 0, L_CONVERGED = 1, L_MAXIT = 2, L_BREAKDOWN = 3, L_NAN = 4 };

struct LState {
    double rho0, alpha, beta, omega1, omega2, rnorm, rnorm0, tol;
    double alpha1, beta1;  // alpha of step 7 and beta of step 11 (the flexible update)
    int k, max_it, done, status, step;
    unsigned int count;
};

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
    dare_gpu::learned::LState* st = nullptr;
    dare_gpu::learned::LState* st_host = nullptr;
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

__device__ __forceinline__ float ahat_apply(const GridDev& g, const float* __restrict__ ah, const float* __restrict__ z,
                                            int64_t c) {
    const int64_t nyz = (int64_t)g.n[1] * g.n[2];
    const int i = (int)(c / nyz), j = (int)((c / g.n[2]) % g.n[1]), k = (int)(c % g.n[2]);
    int64_t nb[7];
    neighbour_ordinals(g, i, j, k, c, nb);
    float v = z[c];
#pragma unroll
    for (int q = 0; q < 6; q++) v += ah[q * g.ncell + c] * z[nb[q + 1]];
    return v;
}

// FP64 r = b - A x -> FP32 rin; ||r||_2 -> *out
__global__ void __launch_bounds__(256) k_residual(GridDev g, const double* __restrict__ diag,
                                                  const double* __restrict__ b, const double* __restrict__ x,
                                                  float* __restrict__ rin, LState* st, double* partials, double* out) {
    const int64_t n = g.ncell, nyz = (int64_t)g.n[1] * g.n[2];
    double acc[1] = {0.};
    GRID_LOOP(c, n) {
        const int i = (int)(c / nyz), j = (int)((c / g.n[2]) % g.n[1]), k = (int)(c % g.n[2]);
        int64_t nb[7];
        neighbour_ordinals(g, i, j, k, c, nb);
        double ax = 0.;
#pragma unroll
        for (int q = 0; q < 7; q++) ax += diag[q * n + c] * x[nb[q]];
        const double r = b[c] - ax;
        rin[c] = (float)r;
        acc[0] += r * r;
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) *out = sqrt(tot[0]);
}

__global__ void __launch_bounds__(256) k_bnorm(int64_t n, const double* __restrict__ b, LState* st, double* partials,
                                               double* out) {
    double acc[1] = {0.};
    GRID_LOOP(c, n) acc[0] += b[c] * b[c];
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) *out = sqrt(tot[0]);
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    GRID_LOOP(c, n) b[c] = (float)a[c];
}

// start of an inner solve: r = rh = rin, u = v = w = d = 0
__global__ void __launch_bounds__(256) k_init(int64_t n, Vecs vs, LState* st, double* partials, double rel_tol,
                                              int max_it) {
    double acc[1] = {0.};
    GRID_LOOP(c, n) {
        const float r = vs.rin[c];
        vs.r[c] = r;
        vs.rh[c] = r;
        vs.u[c] = 0.f;
        vs.v[c] = 0.f;
        vs.w[c] = 0.f;
        vs.d[c] = 0.f;
        acc[0] += (double)r * r;
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
        st->status = L_RUNNING;
        st->step = 0;
        st->done = (st->rnorm0 == 0.) ? 1 : 0;
        if (st->done) st->status = L_CONVERGED;
        if (!(st->rnorm0 == st->rnorm0)) {
            st->done = 1;
            st->status = L_NAN;
        }
    }
}

__device__ __forceinline__ void fail(LState* st, int step) {
    st->done = 1;
    st->status = L_BREAKDOWN;
    st->step = step;
}

// (3), (4): rho1 = <rh, r>, beta
__global__ void __launch_bounds__(256) k_rho(int64_t n, Vecs vs, LState* st, double* partials) {
    if (st->done) return;
    double acc[1] = {0.};
    GRID_LOOP(c, n) acc[0] += (double)vs.rh[c] * vs.r[c];
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
__global__ void k_upd_u(int64_t n, Vecs vs, const LState* st) {
    if (st->done) return;
    const float beta = (float)st->beta;
    GRID_LOOP(c, n) vs.u[c] = vs.r[c] - beta * vs.u[c];
}

// out = Ahat z with <out, rh> (mode 0: gamma -> alpha, steps 7 and 14;
// mode 1: rho1 -> beta, step 11)
__global__ void __launch_bounds__(256) k_spmv_dot(GridDev g, const float* __restrict__ ah, Vecs vs,
                                                  const float* __restrict__ z, float* out, LState* st,
                                                  double* partials, int mode, int step) {
    if (st->done) return;
    double acc[1] = {0.};
    GRID_LOOP(c, g.ncell) {
        const float v = ahat_apply(g, ah, z, c);
        out[c] = v;
        acc[0] += (double)v * vs.rh[c];
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        if (mode == 0) {
            if (tot[0] == 0.) return fail(st, step);
            st->alpha = st->rho0 / tot[0];
            if (step == 7) st->alpha1 = st->alpha;
        } else {
            st->beta = st->alpha * tot[0] / st->rho0;
            st->beta1 = st->beta;
            st->rho0 = tot[0];
        }
    }
}

// (8): r -= alpha v (the matching x update is folded into k_upd_final)
__global__ void k_upd_r(int64_t n, Vecs vs, const LState* st) {
    if (st->done) return;
    const float alpha = (float)st->alpha;
    GRID_LOOP(c, n) vs.r[c] -= alpha * vs.v[c];
}

// (12) v = s - beta v
__global__ void k_upd_v(int64_t n, Vecs vs, const LState* st) {
    if (st->done) return;
    const float beta = (float)st->beta;
    GRID_LOOP(c, n) vs.v[c] = vs.s[c] - beta * vs.v[c];
}

// (15)-(17)
__global__ void k_upd3(int64_t n, Vecs vs, const LState* st) {
    if (st->done) return;
    const float alpha = (float)st->alpha, beta = (float)st->beta;
    GRID_LOOP(c, n) {
        const float r = vs.r[c];
        vs.u[c] = r - beta * vs.u[c];
        vs.r[c] = r - alpha * vs.v[c];
        vs.s[c] -= alpha * vs.w[c];
    }
}

// (18)-(23): t = Ahat z, the five inner products and the omegas
__global__ void __launch_bounds__(256) k_spmv_omega(GridDev g, const float* __restrict__ ah, Vecs vs, LState* st,
                                                    double* partials) {
    if (st->done) return;
    double acc[5] = {0., 0., 0., 0., 0.};
    GRID_LOOP(c, g.ncell) {
        const float t = ahat_apply(g, ah, vs.zs, c);
        vs.t[c] = t;
        const double r = vs.r[c], s = vs.s[c];
        acc[0] += r * s;
        acc[1] += s * s;
        acc[2] += s * t;
        acc[3] += (double)t * t;
        acc[4] += r * t;
    }
    double tot[5];
    if (!grid_reduce<5>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        double om1 = tot[0], mu = tot[1], nu = tot[2], tau = tot[3], om2 = tot[4];
        if (mu == 0.) return fail(st, 20);
        tau -= nu * nu / mu;
        if (tau == 0.) return fail(st, 21);
        om2 = (om2 - nu * om1 / mu) / tau;
        om1 = (om1 - nu * om2) / mu;
        st->omega1 = om1;
        st->omega2 = om2;
    }
}

// (10), (24) in flexible form: d += (a1 - a2 b1) zu + (a2 + w1) zr - w1 a2 zv + w2 zs;
// (25): r -= w1 s + w2 t; u -= w1 v + w2 w; convergence test on ||r||
__global__ void __launch_bounds__(256) k_upd_final(int64_t n, Vecs vs, LState* st, double* partials) {
    if (st->done) return;
    const double a1 = st->alpha1, a2 = st->alpha, b1 = st->beta1, om1 = st->omega1, om2 = st->omega2;
    const float cu = (float)(a1 - a2 * b1), cr = (float)(a2 + om1), cv = (float)(-om1 * a2), cs = (float)om2;
    const float w1 = (float)om1, w2 = (float)om2;
    double acc[1] = {0.};
    GRID_LOOP(c, n) {
        const float r = vs.r[c], s = vs.s[c];
        vs.d[c] += cu * vs.zu[c] + cr * vs.zr[c] + cv * vs.zv[c] + cs * vs.zs[c];
        const float rn = r - w1 * s - w2 * vs.t[c];
        vs.r[c] = rn;
        vs.u[c] -= w1 * vs.v[c] + w2 * vs.w[c];
        acc[0] += (double)rn * rn;
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        const double rn = sqrt(tot[0]);
        st->rnorm = rn;
        if (!(rn == rn)) {
            st->done = 1;
            st->status = L_NAN;
        } else if (rn <= st->tol) {
            st->done = 1;
            st->status = L_CONVERGED;
        } else if (++st->k > st->max_it) {
            st->done = 1;
            st->status = L_MAXIT;
        }
    }
}

// x += D^-1 z (FP64)
__global__ void k_correct(int64_t n, const double* __restrict__ invd, const float* __restrict__ z,
                          double* __restrict__ x) {
    GRID_LOOP(c, n) x[c] += invd[c] * (double)z[c];
}

__global__ void k_to_precond_var(int64_t n, const double* __restrict__ dc, double* __restrict__ x) {
    GRID_LOOP(c, n) x[c] = dc[c] * x[c];
}

static int launch_iteration(dare_ctx* ctx, dare_unet* net, const GridDev& g, const float* ah, const Vecs& vs,
                            LState* st, double* partials) {
    const int64_t n = g.ncell;
    const int eb = grid_blocks(ctx, n, 256, 8);
    cudaStream_t s = ctx->stream;
    int rc;
    k_rho<<<eb, 256, 0, s>>>(n, vs, st, partials);
    DARE_LAUNCHED(ctx);
    k_upd_u<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.u, vs.zu))) return rc;
    k_spmv_dot<<<eb, 256, 0, s>>>(g, ah, vs, vs.zu, vs.v, st, partials, 0, 7);
    DARE_LAUNCHED(ctx);
    k_upd_r<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.r, vs.zr))) return rc;
    k_spmv_dot<<<eb, 256, 0, s>>>(g, ah, vs, vs.zr, vs.s, st, partials, 1, 11);
    DARE_LAUNCHED(ctx);
    k_upd_v<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.v, vs.zv))) return rc;
    k_spmv_dot<<<eb, 256, 0, s>>>(g, ah, vs, vs.zv, vs.w, st, partials, 0, 14);
    DARE_LAUNCHED(ctx);
    k_upd3<<<eb, 256, 0, s>>>(n, vs, st);
    DARE_LAUNCHED(ctx);
    if ((rc = unet::apply(net, vs.s, vs.zs))) return rc;
    k_spmv_omega<<<eb, 256, 0, s>>>(g, ah, vs, st, partials);
    DARE_LAUNCHED(ctx);
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
    if (g.dim != 3 || g.n[0] != net->n[0] || g.n[1] != net->n[1] || g.n[2] != net->n[2])
        return set_error(ctx, DARE_ERR_BAD_ARG, "bicgstab2_learned: grid does not match the network");
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
        if (e == cudaSuccess) e = cudaMalloc(&lw->st, sizeof(LState));
        if (e == cudaSuccess) e = cudaMemset(lw->st, 0, sizeof(LState));
        if (e == cudaSuccess) e = cudaMallocHost(&lw->st_host, sizeof(LState));
        if (e != cudaSuccess) {
            dare_learned_ws_free(lw);
            return check_cuda(ctx, e, "bicgstab2_learned workspace");
        }
        ws->learned = lw;
    }
    dare_learned_ws* lw = ws->learned;
    const int eb = grid_blocks(ctx, n, 256, 8);
    float* V = lw->vec;
    Vecs vs;
    float** slots[kNumVecs] = {&vs.rh, &vs.r, &vs.u, &vs.v, &vs.s, &vs.w, &vs.t,
                               &vs.d, &vs.zu, &vs.zr, &vs.zv, &vs.zs, &vs.rin};
    for (int i = 0; i < kNumVecs; i++) *slots[i] = V + (size_t)i * n;

    // Ahat = A D^-1 (FP64 fold) and its FP32 copy
    if ((rc = launch_fold(ctx, g, ws->march, s->diag, ws->invd, ws->ahat, ws->st, ws->partials))) return rc;
    k_to_f32<<<eb, 256, 0, ctx->stream>>>(ws->ahat, lw->ahat32, 6 * n);
    DARE_LAUNCHED(ctx);
    DARE_CUDA(ctx, cudaMemsetAsync(lw->st, 0, sizeof(LState), ctx->stream));
    k_bnorm<<<eb, 256, 0, ctx->stream>>>(n, s->rhs, lw->st, lw->partials, lw->scal);
    DARE_LAUNCHED(ctx);
    double bnorm = 0.;
    if ((rc = read_scalar(ctx, lw->scal, &bnorm))) return rc;
    const double tol_abs = p->tol_relative ? p->tol * bnorm : p->tol;

    // one CUDA graph per inner iteration (captured once per network and system)
    if (!lw->graph || lw->graph_net != net) {
        if (lw->graph) cudaGraphExecDestroy(lw->graph);
        lw->graph = nullptr;
        if ((rc = dare_gpu::unet::apply(net, vs.rin, vs.zs))) return rc;  // sets the launch configurations
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaGraph_t graph = nullptr;
        DARE_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = ctx->launches;
        rc = launch_iteration(ctx, net, g, lw->ahat32, vs, lw->st, lw->partials);
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
    for (int it = 0;; it++) {
        k_residual<<<eb, 256, 0, ctx->stream>>>(g, s->diag, s->rhs, s->x, vs.rin, lw->st, lw->partials, lw->scal);
        DARE_LAUNCHED(ctx);
        if ((rc = read_scalar(ctx, lw->scal, &rnorm))) return rc;
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
            DARE_CUDA(ctx, cudaMemcpyAsync(lw->st_host, lw->st, sizeof(LState), cudaMemcpyDeviceToHost, ctx->stream));
            DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (lw->st_host->done) break;
        }
        DARE_CUDA(ctx, cudaMemcpyAsync(lw->st_host, lw->st, sizeof(LState), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        const LState st = *lw->st_host;
        inner_total += std::min(st.k, cap);
        if (st.status == L_NAN) break;
        // x += D^-1 d
        k_correct<<<eb, 256, 0, ctx->stream>>>(n, ws->invd, vs.d, s->x);
        DARE_LAUNCHED(ctx);
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
