// dare_mixed.cu -- FP32-inner / FP64-refinement BiCGStab(2).
//
// The Krylov bulk (SpMV, axpys, the folded Jacobi preconditioner) runs in
// FP32 on an FP32 copy of Ahat = A D^-1, while every dot product that sets
// alpha / omega and the breakdown checks accumulates in FP64 (the fused
// kernels reduce in double).  The outer loop is FP64 iterative refinement:
//     r = b - A x          (FP64, the assembled operator; also the stop test)
//     Ahat dy = r          (FP32 BiCGStab2 to a relative tolerance)
//     x += D^-1 dy         (FP64)
// until ||b - A x||_2 <= tol.  If the correction stops contracting, the
// driver falls back to the plain FP64 solve from the current iterate.
// Per inner iteration the FP32 kernels move about half the bytes of FP64.
#include <cmath>
#include <cstring>

#include "dare_march.cuh"

using namespace dare_gpu;

void dare_mixed_ws_free(dare_solver_ws* ws) {
    if (!ws) return;
    cudaFree(ws->ahat32);
    cudaFree(ws->vec32);
    cudaFree(ws->r64);
    ws->ahat32 = nullptr;
    ws->vec32 = nullptr;
    ws->r64 = nullptr;
}

namespace dare_gpu {


// x += D^-1 dy
static __global__ void k_correct(int64_t n, const double* __restrict__ invd, const float* __restrict__ dy,
                                 double* __restrict__ x) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        x[c] = invd[c] * (double)dy[c] + x[c];
}

// y = D x (continue the FP64 solve from the current iterate in its variable)
static __global__ void k_to_precond_var(int64_t n, const double* __restrict__ dc, double* __restrict__ x) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        x[c] = dc[c] * x[c];
}

// ||b||^2 -> *out (sqrt)
static __global__ void __launch_bounds__(256) k_norm(int64_t n, const double* __restrict__ b, SolverState* st,
                                                     double* partials, double* out) {
    double acc[1] = {0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        acc[0] += b[c] * b[c];
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) *out = sqrt(tot[0]);
}

// r = b - A x in FP64; r32 = (float) r; dy = 0; ||r||_2 -> *out
struct FRefResidual {
    using type = double;
    static constexpr int Q = 1, NZ = 1, NP = 8;
    static constexpr bool kCheckDone = false;
    static constexpr bool kPairs = false;
    const double* zs[2];   // x
    const double* ps[NP];  // 7 coefficients, b
    float* r32;
    float* dy;
    double* out;
    __device__ void load(const SolverState*) {}
    __device__ double zc(double a, double) const { return a; }
    __device__ void center(int64_t c, const double (&zz)[7], const double* p, double* acc) const {
        const double r = p[7] - apply_pre<double, false>(p, zz);
        r32[c] = (float)r;
        dy[c] = 0.f;
        acc[0] += r * r;
    }
    __device__ void done(SolverState*, const double* tot) const { *out = sqrt(tot[0]); }
};

static int read_scalar(dare_ctx* ctx, const double* dptr, double* out) {
    DARE_CUDA(ctx, cudaMemcpyAsync(out, dptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

}  // namespace dare_gpu

int dare_bicgstab2_refine(dare_system* s, const dare_solver_params* p, dare_solve_report* rep) {
    using namespace dare_gpu;
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->sdev;   // components stacked along i
    if (p->precond != DARE_PREC_JACOBI)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "FP32 refinement is built for the Jacobi-folded operator");
    int rc = ensure_solver_ws(s);
    if (rc) return rc;
    dare_solver_ws* ws = s->ws;
    const int64_t n = g.ncell;
    if (!ws->ahat32) {
        cudaError_t e = cudaMalloc(&ws->ahat32, (size_t)n * 6 * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&ws->vec32, (size_t)n * 13 * sizeof(float));
        if (e != cudaSuccess) {
            dare_mixed_ws_free(ws);
            return check_cuda(ctx, e, "refinement workspace");
        }
        ws->march32 = march_config(ctx, g, sizeof(float));
    }
    const MarchCfg& m = ws->march;
    const MarchCfg& m32 = ws->march32;
    const int eb = grid_blocks(ctx, n, 256, 8);
    OpT<double> full{s->diag, s->diag + n, n};

    // Ahat = A D^-1, folded straight to FP32
    if ((rc = launch_fold32(ctx, g, m, s->diag, ws->invd, ws->ahat32, ws->st, ws->partials))) return rc;
    OpT<float> op32{nullptr, ws->ahat32, n};
    float* dy = ws->vec32 + 11 * n;
    float* r32 = ws->vec32 + 12 * n;
    VecsT<float> vs32 = carve_vecs<float>(ws->vec32, n, dy, r32);

    double* scratch = ws->partials + (size_t)kMaxQ * kMaxBlocks;
    SolverState zero{};
    DARE_CUDA(ctx, cudaMemcpyAsync(ws->st, &zero, sizeof(zero), cudaMemcpyHostToDevice, ctx->stream));
    k_norm<<<eb, 256, 0, ctx->stream>>>(n, s->rhs, ws->st, ws->partials, scratch);
    DARE_LAUNCHED(ctx);
    double bnorm = 0.;
    if ((rc = read_scalar(ctx, scratch, &bnorm))) return rc;
    const double tol_abs = p->tol_relative ? p->tol * bnorm : p->tol;

    std::memset(rep, 0, sizeof(*rep));
    rep->b_norm = bnorm;
    rep->tol_abs = tol_abs;
    double rnorm = 0., prev = INFINITY;
    bool converged = false;
    int refinements = 0, inner_total = 0;
    for (int it = 0; it <= p->max_refinements; it++) {
        FRefResidual fr{};
        fr.zs[0] = s->x;
        set_coef_streams<double, false, 8>(full, fr.ps);
        fr.ps[7] = s->rhs;
        fr.r32 = r32;
        fr.dy = dy;
        fr.out = scratch;
        if ((rc = launch_march(ctx, g, m, fr, ws->st, ws->partials))) return rc;
        if ((rc = read_scalar(ctx, scratch, &rnorm))) return rc;
        if (rnorm <= tol_abs) {
            converged = true;
            break;
        }
        if (!(rnorm < 0.5 * prev) || it == p->max_refinements) {  // not contracting (or NaN)
            break;
        }
        prev = rnorm;
        // inner FP32 BiCGStab2 on Ahat dy = r, relative tolerance, FP64 dots
        SolverState init{};
        init.tol = p->inner_rel_tol;
        init.tol_relative = 1;
        init.max_it = p->inner_max_it;
        DARE_CUDA(ctx, cudaMemcpyAsync(ws->st, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = launch_init<float, true>(ctx, g, m32, op32, vs32, ws->st, ws->partials))) return rc;
        if ((rc = run_iterations<float, true>(ctx, g, m32, ws->stream_blocks, op32, vs32, ws->st, ws->st_host,
                                              ws->partials, &ws->graph[2][0], p->inner_max_it, p->check_every, 9)))
            return rc;
        inner_total += ws->st_host->k;
        if (ws->st_host->status == ST_NAN) {
            break;
        }
        if ((rc = finish_step10(ctx, n, *ws->st_host, ws->st, vs32))) return rc;
        k_correct<<<eb, 256, 0, ctx->stream>>>(n, ws->invd, dy, s->x);
        DARE_LAUNCHED(ctx);
        refinements++;
    }
    rep->refinements = refinements;
    rep->inner_iters = inner_total;
    rep->iters = inner_total;
    rep->res_abs = rnorm;
    if (converged) {
        rep->converged = 1;
        rep->status = DARE_SOLVE_CONVERGED;
        rep->true_res_abs = rnorm;
        return DARE_OK;
    }
    // fallback: the plain FP64 solve from the current iterate (y = D x)
    k_to_precond_var<<<eb, 256, 0, ctx->stream>>>(n, s->diag, s->x);
    DARE_LAUNCHED(ctx);
    dare_solver_params q = *p;
    q.precision = DARE_PRECISION_FP64;
    q.tol = tol_abs;
    q.tol_relative = 0;
    dare_solve_report r2;
    if ((rc = dare_bicgstab2_fp64(s, &q, &r2))) return rc;
    *rep = r2;
    rep->refinements = refinements;
    rep->inner_iters = inner_total;
    rep->fallback_used = 1;
    rep->b_norm = bnorm;
    return DARE_OK;
}
