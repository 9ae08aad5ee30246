// dare_bicgstab2.cu -- device-resident BiCGStab(2) for the structured
// 7-point systems (MatrixSystem/BiCGStab2.inl:166-582, van der Vorst's
// unrolled Sleijpen-Fokkema form, right preconditioner).
//
// Design (HBM-bound; every kernel streams its operands once):
//   * Jacobi is folded into the operator: Ahat = A D^-1 (column scaling), so
//     Ahat has a unit diagonal and each SpMV reads 6 off-diagonals.  The
//     iteration runs in the preconditioned variable y (x = D^-1 y), exactly
//     as the reference: r0 = b - A M^-1 x_init, x = M^-1 y at the end.
//   * One iteration = 5 kernels.  Four of them fuse the axpy that produces an
//     SpMV input with the SpMV and the dot products after it.  They are
//     plane-marching stencil kernels: a block owns a (j,k) tile, walks along i
//     keeping the fused input of planes i-1, i, i+1 in registers and plane i
//     (with its j/k halo) in shared memory, so each operand is read from HBM
//     once and each fused value is evaluated once per cell (plus the halo).
//     Each of r, u, v and s has a second buffer for the value of the middle
//     of an iteration: step (10), x += alpha u, and step (15),
//     u = r - beta u, wait for the last kernel, which reads both buffers.
//     A graph holds two iterations.
//   * Scalars (alpha, beta, rho, omega, ...) never leave the device: the last
//     block of each kernel reduces the per-block partials in a fixed order
//     (deterministic, no floating-point atomics), evaluates the reference's
//     scalar recurrence and its breakdown checks, and sets a done flag that
//     turns every later kernel into a no-op.  The host polls that flag.
//   * The reference keeps omega/mu/nu/tau in long double; here they are FP64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "dare_march.cuh"

using namespace dare_gpu;

void dare_solver_ws_free(dare_solver_ws* ws) {
    if (!ws) return;
    for (auto& row : ws->graph)
        for (auto& g : row)
            if (g) cudaGraphExecDestroy(g);
    cudaFree(ws->ahat);
    cudaFree(ws->invd);
    cudaFree(ws->vec);
    cudaFree(ws->partials);
    cudaFree(ws->st);
    if (ws->st_host) cudaFreeHost(ws->st_host);
    dare_mixed_ws_free(ws);
    dare_learned_ws_free(ws->learned);
    delete ws;
}

namespace dare_gpu {

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
MarchCfg march_config(const dare_ctx* ctx, const GridDev& g, size_t elem, int max_items) {
    MarchCfg m;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    int tk = n2 > 16 ? 32 : n2 > 8 ? 16 : n2 > 4 ? 8 : n2 > 2 ? 4 : 1;
    int tj = 256 / tk;
    if (n2 % 2 == 0 && n2 >= 32) {
        // two cells per thread: 16 x 8 threads on 32 x 8 cells (the same
        // tile and shared memory as one cell per thread, half the threads)
        m.cpt = 2;
        tk = 16;
        tj = 8;
    }
    if (elem == 4 && n2 % 4 == 0 && n2 >= 64) {
        // FP32: four cells per thread, 16 x 8 threads on 64 x 8 cells (every
        // row segment one 16-byte copy)
        m.cpt = 4;
        tk = 16;
        tj = 8;
    }
    while (tj > 1 && tj / 2 >= n1) tj /= 2;
    m.block = dim3(tk, tj, 1);
    m.tiles_x = (n2 + tk * m.cpt - 1) / (tk * m.cpt);
    m.tiles_y = (n1 + tj - 1) / tj;
    const int64_t tiles = (int64_t)m.tiles_x * m.tiles_y;
    // Longest plane run that still leaves ~4 items per resident block (the
    // dynamic queue then ends with a short tail); each run re-reads 2 planes.
    // With several field components (stacked along i) runs stay inside one.
    const int nc = g.ncomp, n0c = n0 / nc;
    const int64_t want = (int64_t)ctx->num_sms * 3 * 4;
    int planes = 32;
    while (planes > 4 && tiles * nc * ((n0c + planes - 1) / planes) < want) planes /= 2;
    while (tiles * nc * ((n0c + planes - 1) / planes) > max_items && planes < n0c) planes *= 2;
    if (planes > n0c) planes = n0c;
    m.planes = planes;
    m.cpc = (n0c + planes - 1) / planes;
    m.nitems = (int)(tiles * nc * m.cpc);
    m.smem = 2 * (size_t)(tk * m.cpt + 2) * (tj + 2) * elem;
    return m;
}

int ensure_solver_ws(dare_system* s) {
    dare_ctx* ctx = s->grid->ctx;
    const int64_t n = s->sdev.ncell;   // all field components
    if (s->ws && s->ws->n == n) return DARE_OK;
    dare_solver_ws_free(s->ws);
    s->ws = nullptr;
    dare_solver_ws* ws = new (std::nothrow) dare_solver_ws();
    if (!ws) return DARE_ERR_OOM;
    ws->n = n;
    cudaError_t e = cudaMalloc(&ws->ahat, (size_t)n * 6 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->invd, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->vec, (size_t)n * 11 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->partials, (size_t)kMaxQ * kMaxBlocks * sizeof(double) + 64);
    if (e == cudaSuccess) e = cudaMalloc(&ws->st, sizeof(SolverState));
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->st, 0, sizeof(SolverState), ctx->stream);
    if (e == cudaSuccess) e = cudaMallocHost(&ws->st_host, sizeof(SolverState));
    if (e != cudaSuccess) {
        dare_solver_ws_free(ws);
        return check_cuda(ctx, e, "bicgstab2 workspace");
    }
    ws->march = march_config(ctx, s->sdev, sizeof(double));
    ws->stream_blocks = grid_blocks(ctx, n, 256, 8);
    s->ws = ws;
    return DARE_OK;
}

template <typename T>
VecsT<T> carve_vecs(T* base, int64_t n, T* x, const T* b) {
    VecsT<T> v;
    v.x = x;
    v.b = b;
    v.rh = base;
    v.r[0] = base + 1 * n;
    v.r[1] = base + 2 * n;
    v.u[0] = base + 3 * n;
    v.u[1] = base + 4 * n;
    v.v[0] = base + 5 * n;
    v.v[1] = base + 6 * n;
    v.s[0] = base + 7 * n;
    v.s[1] = base + 8 * n;
    v.w = base + 9 * n;
    v.t = base + 10 * n;
    return v;
}
template VecsT<double> carve_vecs<double>(double*, int64_t, double*, const double*);
template VecsT<float> carve_vecs<float>(float*, int64_t, float*, const float*);

template <typename T, bool UNIT>
int launch_init(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const OpT<T>& op, const VecsT<T>& vs,
                SolverState* st, double* partials) {
    return launch_march(ctx, g, m, make_init<T, UNIT>(op, vs), st, partials);
}
template int launch_init<double, true>(dare_ctx*, const GridDev&, const MarchCfg&, const OpT<double>&,
                                       const VecsT<double>&, SolverState*, double*);
template int launch_init<double, false>(dare_ctx*, const GridDev&, const MarchCfg&, const OpT<double>&,
                                        const VecsT<double>&, SolverState*, double*);
template int launch_init<float, true>(dare_ctx*, const GridDev&, const MarchCfg&, const OpT<float>&,
                                      const VecsT<float>&, SolverState*, double*);

// One iteration (`par`: its place in the pair a graph holds; every iteration
// uses the same buffers).  `ev` (optional, profiling): ev[0] before the first
// kernel, ev[1..5] after each.
template <typename T, bool UNIT>
int launch_iteration(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, int sblocks, const OpT<T>& op,
                     const VecsT<T>& vs, SolverState* st, double* partials, int par, cudaEvent_t* ev) {
    (void)par;
    cudaStream_t sm = ctx->stream;
    int rc;
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[0], sm));
    if ((rc = launch_march(ctx, g, m, make_step1<T, UNIT>(op, vs), st, partials))) return rc;
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[1], sm));
    if ((rc = launch_march(ctx, g, m, make_step2<T, UNIT>(op, vs), st, partials))) return rc;
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[2], sm));
    if ((rc = launch_march(ctx, g, m, make_step3<T, UNIT>(op, vs), st, partials))) return rc;
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[3], sm));
    if ((rc = launch_march(ctx, g, m, make_step4<T, UNIT>(op, vs), st, partials))) return rc;
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[4], sm));
    int vec4 = 0;
    if constexpr (sizeof(T) == 4) {
        const void* arrs[10] = {vs.x, vs.r[0], vs.s[1], vs.t, vs.u[0], vs.u[1], vs.r[1], vs.v[1], vs.w, vs.rh};
        vec4 = g.ncell % 4 == 0;
        for (const void* a : arrs)
            if (a && reinterpret_cast<uintptr_t>(a) % 16 != 0) vec4 = 0;
    }
    k_step5<T><<<sblocks, 256, 0, sm>>>(g.ncell, vs.x, vs.r[0], vs.s[1], vs.t, vs.u[0], vs.u[1], vs.r[1], vs.v[1],
                                        vs.w, vs.rh, st, partials, 0, 0, vec4);
    DARE_LAUNCHED(ctx);
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[5], sm));
    return DARE_OK;
}
template int launch_iteration<double, true>(dare_ctx*, const GridDev&, const MarchCfg&, int, const OpT<double>&,
                                            const VecsT<double>&, SolverState*, double*, int, cudaEvent_t*);
template int launch_iteration<double, false>(dare_ctx*, const GridDev&, const MarchCfg&, int, const OpT<double>&,
                                             const VecsT<double>&, SolverState*, double*, int, cudaEvent_t*);
template int launch_iteration<float, true>(dare_ctx*, const GridDev&, const MarchCfg&, int, const OpT<float>&,
                                           const VecsT<float>&, SolverState*, double*, int, cudaEvent_t*);

int launch_true_residual(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const OpT<double>& op,
                         const double* x, const double* b, SolverState* st, double* partials, double* out) {
    return launch_march(ctx, g, m, make_residual(op, x, b, out), st, partials);
}

int launch_fold(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const double* diag, double* invd, double* ahat,
                SolverState* st, double* partials) {
    const int eb = grid_blocks(ctx, g.ncell, 256, 8);
    k_invdiag<<<eb, 256, 0, ctx->stream>>>(diag, invd, g.ncell);
    DARE_LAUNCHED(ctx);
    return launch_march(ctx, g, m, make_fold(diag, invd, ahat, g.ncell), st, partials);
}

// invd = 1 / diag, then the fold and the init kernel in one pass (FFoldInit)
int launch_fold_init(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const double* diag, double* invd,
                     double* ahat, const VecsT<double>& vs, SolverState* st, double* partials) {
    const int64_t n = g.ncell;
    k_invdiag<<<grid_blocks(ctx, n, 256, 8), 256, 0, ctx->stream>>>(diag, invd, n);
    DARE_LAUNCHED(ctx);
    FFoldInit f{};
    f.zs[0] = invd;
    f.zs[1] = vs.x;
    for (int q = 0; q < 6; q++) f.ps[q] = diag + (q + 1) * n;
    f.ps[6] = vs.b;
    f.ahat = ahat;
    f.r = vs.r[0];
    f.rh = vs.rh;
    f.u = vs.u[0];
    f.n = n;
    return launch_march(ctx, g, m, f, st, partials);
}

int launch_fold32(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const double* diag, double* invd, float* ahat32,
                  SolverState* st, double* partials) {
    const int eb = grid_blocks(ctx, g.ncell, 256, 8);
    k_invdiag<<<eb, 256, 0, ctx->stream>>>(diag, invd, g.ncell);
    DARE_LAUNCHED(ctx);
    FFold32 f{};
    f.zs[0] = invd;
    for (int q = 0; q < 6; q++) f.ps[q] = diag + (q + 1) * g.ncell;
    f.ahat = ahat32;
    f.n = g.ncell;
    return launch_march(ctx, g, m, f, st, partials);
}

template <typename T>
int finish_step10(dare_ctx* ctx, int64_t n, const SolverState& st_host, const SolverState* st, const VecsT<T>& vs) {
    if (!step10_pending(st_host)) return DARE_OK;
    k_step10<T><<<grid_blocks(ctx, n, 256, 8), 256, 0, ctx->stream>>>(n, st, vs.u[1], vs.x);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}
template int finish_step10<double>(dare_ctx*, int64_t, const SolverState&, const SolverState*, const VecsT<double>&);
template int finish_step10<float>(dare_ctx*, int64_t, const SolverState&, const SolverState*, const VecsT<float>&);

int launch_scale(dare_ctx* ctx, int64_t n, const double* invd, double* x) {
    const int eb = grid_blocks(ctx, n, 256, 8);
    k_scale<<<eb, 256, 0, ctx->stream>>>(n, invd, x);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// Read the solver state back after the iterations; a state that is not done
// means the bound was reached without a status.
int finish_iterations(dare_ctx* ctx, const SolverState* st, SolverState* st_host) {
    DARE_CUDA(ctx, cudaMemcpyAsync(st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!st_host->done) return set_error(ctx, DARE_ERR_STATE, "bicgstab2: iteration bound reached without a status");
    return DARE_OK;
}

// Two iterations captured as one CUDA graph.  (A device-side loop, a
// conditional WHILE node around them, was measured as well: no faster on
// the boxes measured, and ncu does not profile kernels of graphs that can
// hold conditional nodes, so the host replays this graph and polls.)
template <typename T, bool UNIT>
static int build_graph(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, int sblocks, const OpT<T>& op,
                       const VecsT<T>& vs, SolverState* st, double* partials, cudaGraphExec_t* out) {
    cudaStream_t cap;
    DARE_CUDA(ctx, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaStream_t saved = ctx->stream;
    ctx->stream = cap;
    cudaGraph_t graph = nullptr;
    int rc = DARE_OK;
    const int64_t launches0 = ctx->launches;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = launch_iteration<T, UNIT>(ctx, g, m, sblocks, op, vs, st, partials, 0, nullptr);
        if (rc == DARE_OK) rc = launch_iteration<T, UNIT>(ctx, g, m, sblocks, op, vs, st, partials, 1, nullptr);
        cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
        if (e == cudaSuccess) e = e2;
    }
    ctx->stream = saved;
    ctx->launches = launches0;  // captured, not executed
    if (e == cudaSuccess && rc == DARE_OK) e = cudaGraphInstantiate(out, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != DARE_OK) return rc;
    if (e != cudaSuccess) return check_cuda(ctx, e, "bicgstab2 graph capture");
    return DARE_OK;
}

// Run iterations until the done flag is set: replays of the two-iteration
// graph, the state read back every `check_every` pairs (0: by grid size), or,
// when profiling, direct launches with per-kernel events and a read after
// every pair.  `wait`: read the final state back again before returning
// (otherwise the caller queues more work and reads it with the state).
template <typename T, bool UNIT>
int run_iterations(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, int sblocks, const OpT<T>& op,
                   const VecsT<T>& vs, SolverState* st, SolverState* st_host, double* partials, cudaGraphExec_t* ge,
                   int max_it, int check_every, int kid_base, bool wait) {
    const bool prof = ctx->profiling != 0;
    const int max_pairs = max_it / 2 + 2;
    if (!prof) {
        if (!*ge) {
            int rc = build_graph<T, UNIT>(ctx, g, m, sblocks, op, vs, st, partials, ge);
            if (rc) return rc;
        }
        if (check_every <= 0) {
            const int64_t per = (int64_t)1 << 21;
            check_every = (int)std::min<int64_t>(8, std::max<int64_t>(1, (per + g.ncell - 1) / g.ncell));
        }
        for (int gi = 0; gi < max_pairs; gi++) {
            DARE_CUDA(ctx, cudaGraphLaunch(*ge, ctx->stream));
            ctx->launches += 10;
            if ((gi + 1) % check_every == 0 || gi + 1 == max_pairs) {
                DARE_CUDA(ctx, cudaMemcpyAsync(st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                               ctx->stream));
                DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
                if (st_host->done) break;
            }
        }
        if (!wait) return st_host->done ? DARE_OK
                                        : set_error(ctx, DARE_ERR_STATE,
                                                    "bicgstab2: iteration bound reached without a status");
        return finish_iterations(ctx, st, st_host);
    }
    // profiling checks after every pair, so each recorded duration belongs
    // to a known iteration
    for (int gi = 0; gi < max_pairs; gi++) {
        for (int par = 0; par < 2; par++) {
            int rc = launch_iteration<T, UNIT>(ctx, g, m, sblocks, op, vs, st, partials, par, ctx->ev + 5 * par);
            if (rc) return rc;
        }
        DARE_CUDA(ctx, cudaMemcpyAsync(st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        // Iterations of this pair that ran in full: both while the
        // solve goes on; on convergence the flag is raised by the
        // last kernel of iteration k (k = 2 gi + 1 or 2 gi + 2), and
        // the kernels after it returned at once.  A pair that ended
        // in another status is not recorded.
        int real = 2;
        if (st_host->done) {
            real = st_host->status == ST_CONVERGED ? st_host->k - 2 * gi : 0;
            real = real < 0 ? 0 : real > 2 ? 2 : real;
        }
        for (int it = 0; it < real; it++)
            for (int q = 0; q < 5; q++) {
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, ctx->ev[it * 5 + q], ctx->ev[it * 5 + q + 1]) == cudaSuccess) {
                    ctx->stat_ms[kid_base + q] += ms;
                    ctx->stat_n[kid_base + q] += 1;
                } else {
                    cudaGetLastError();  // timing is best effort; do not leak the error
                }
            }
        if (st_host->done) break;
    }
    return finish_iterations(ctx, st, st_host);
}
template int run_iterations<float, true>(dare_ctx*, const GridDev&, const MarchCfg&, int, const OpT<float>&,
                                         const VecsT<float>&, SolverState*, SolverState*, double*, cudaGraphExec_t*,
                                         int, int, int, bool);

}  // namespace dare_gpu

namespace dare_gpu {
bool solution_to_field_ok(const GridDev& g);
int launch_solution_to_field(dare_ctx* ctx, const GridDev& g, const double* invd, double* x, double* phi);
}  // namespace dare_gpu

// Plain FP64 solve (BiCGStab2::Solve on the device).  With a field `f` (the
// time step's), the exit's x = M^-1 y also writes x into the field's level 0
// with its periodic face ghosts (CopyTo and ExchangeHaloCells in the same
// pass); *field_written says whether the field holds the returned x.
int dare_bicgstab2_fp64_to(dare_system* s, const dare_solver_params* p, dare_solve_report* rep, dare_field* f,
                           int* field_written) {
    using namespace dare_gpu;
    if (field_written) *field_written = 0;
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->sdev;   // components stacked along i
    int rc = ensure_solver_ws(s);
    if (rc) return rc;
    dare_solver_ws* ws = s->ws;
    const int64_t n = g.ncell;
    const bool jacobi = p->precond == DARE_PREC_JACOBI;
    const MarchCfg& m = ws->march;

    OpT<double> full{s->diag, s->diag + n, n};
    OpT<double> folded{nullptr, ws->ahat, n};
    SolverState init{};   // also zeroes the reduction and queue counters
    init.tol = p->tol;
    init.max_it = p->max_it;
    init.tol_relative = p->tol_relative;
    DARE_CUDA(ctx, cudaMemcpyAsync(ws->st, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    VecsT<double> vs = carve_vecs<double>(ws->vec, n, s->x, s->rhs);
    rc = jacobi ? launch_fold_init(ctx, g, m, s->diag, ws->invd, ws->ahat, vs, ws->st, ws->partials)
                : launch_init<double, false>(ctx, g, m, full, vs, ws->st, ws->partials);
    if (rc) return rc;
    rc = jacobi ? run_iterations<double, true>(ctx, g, m, ws->stream_blocks, folded, vs, ws->st, ws->st_host,
                                               ws->partials, &ws->graph[1][0], p->max_it, p->check_every, KID_STEP1,
                                               false)
                : run_iterations<double, false>(ctx, g, m, ws->stream_blocks, full, vs, ws->st, ws->st_host,
                                                ws->partials, &ws->graph[0][0], p->max_it, p->check_every, KID_STEP1,
                                                false);
    if (rc) return rc;
    // The exit's device work, queued behind the iterations and read back with
    // the state in one round trip: step (10) when the solve stopped after it
    // (decided on the device), x = M^-1 y, and the true residual of that x
    // (the report's, and the tau = 0 exit's check).
    k_step10<double><<<grid_blocks(ctx, n, 256, 8), 256, 0, ctx->stream>>>(n, ws->st, vs.u[1], vs.x);
    DARE_LAUNCHED(ctx);
    const GridDev& gf = s->grid->dev;   // one field component
    const bool to_field = f && field_written && f->grid == s->grid && f->ncomp == s->ncomp && solution_to_field_ok(gf);
    if (to_field) {
        for (int c = 0; c < s->ncomp; c++)
            if ((rc = launch_solution_to_field(ctx, gf, jacobi ? ws->invd + (size_t)c * gf.ncell : nullptr,
                                               s->x + (size_t)c * gf.ncell, f->level[0] + (size_t)c * gf.ncell_ghosted)))
                return rc;
    } else if (jacobi && (rc = launch_scale(ctx, n, ws->invd, s->x))) {
        return rc;
    }
    bool field_current = to_field;
    double* tres = &ws->st->tres;
    if (p->compute_true_residual &&
        (rc = launch_true_residual(ctx, g, m, full, s->x, s->rhs, ws->st, ws->partials, tres)))
        return rc;
    if ((rc = finish_iterations(ctx, ws->st, ws->st_host))) return rc;
    SolverState st = *ws->st_host;

    std::memset(rep, 0, sizeof(*rep));
    rep->iters = st.k;
    rep->b_norm = sqrt(st.bnorm2);
    rep->res_abs = st.rnorm;
    rep->breakdown_step = st.step;
    rep->tol_abs = st.tol;
    if (p->compute_true_residual) rep->true_res_abs = st.tres;
    if (st.status == ST_TAU0) {
        // BiCGStab2.inl:407-424: x = M^-1 y, true residual, return if converged;
        // otherwise break to the common exit, which applies M^-1 once more.
        double tr = st.tres;
        if (!p->compute_true_residual) {
            if ((rc = launch_true_residual(ctx, g, m, full, s->x, s->rhs, ws->st, ws->partials, tres))) return rc;
            if ((rc = finish_iterations(ctx, ws->st, ws->st_host))) return rc;
            tr = ws->st_host->tres;
        }
        rep->res_abs = tr;
        if (tr <= st.tol) {
            rep->converged = 1;
            rep->status = DARE_SOLVE_CONVERGED;
            rep->breakdown_step = 0;
        } else {
            rep->converged = 0;
            rep->status = DARE_SOLVE_BREAKDOWN;
            if (jacobi) {
                if ((rc = launch_scale(ctx, n, ws->invd, s->x))) return rc;
                field_current = false;   // x changed after the field was written
                if (p->compute_true_residual) {
                    if ((rc = launch_true_residual(ctx, g, m, full, s->x, s->rhs, ws->st, ws->partials, tres)))
                        return rc;
                    if ((rc = finish_iterations(ctx, ws->st, ws->st_host))) return rc;
                    rep->true_res_abs = ws->st_host->tres;
                }
            }
        }
    } else {
        rep->converged = st.rnorm <= st.tol;
        switch (st.status) {
        case ST_CONVERGED: rep->status = DARE_SOLVE_CONVERGED; break;
        case ST_MAXIT: rep->status = DARE_SOLVE_MAXIT; break;
        case ST_NAN: rep->status = DARE_SOLVE_NAN; break;
        default: rep->status = DARE_SOLVE_BREAKDOWN; break;
        }
    }
    if (field_written) *field_written = field_current ? 1 : 0;
    return DARE_OK;
}

int dare_bicgstab2_fp64(dare_system* s, const dare_solver_params* p, dare_solve_report* rep) {
    return dare_bicgstab2_fp64_to(s, p, rep, nullptr, nullptr);
}

int dare_bicgstab2_refine(dare_system* s, const dare_solver_params* p, dare_solve_report* rep);

extern "C" {

void dare_solver_params_default(dare_solver_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->tol = 1e-8;         // BiCGStab2 constructor defaults (BiCGStab2.inl:29-31)
    p->max_it = 100;
    p->precond = DARE_PREC_JACOBI;
    p->precision = DARE_PRECISION_FP64;
    p->inner_rel_tol = 1e-5;
    p->inner_max_it = 200;
    p->max_refinements = 30;
    p->check_every = 0;
    p->compute_true_residual = 1;
}

// dare_bicgstab2_solve for a time step of field f: with the plain FP64
// solve, the field is written at the solve's exit (*field_written = 1);
// otherwise the caller copies x into it.
int dare_bicgstab2_solve_to_field(dare_system* s, const dare_solver_params* p, dare_solve_report* rep,
                                  dare_field* f, int* field_written) {
    *field_written = 0;
    if (!s || !p || !rep) return DARE_ERR_BAD_ARG;
    if (p->max_it < 0 || !(p->tol >= 0.)) return dare_gpu::set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "bicgstab2: bad params");
    if (p->precond != DARE_PREC_NONE && p->precond != DARE_PREC_JACOBI)
        return dare_gpu::set_error(s->grid->ctx, DARE_ERR_UNSUPPORTED, "bicgstab2: preconditioner not supported");
    cudaSetDevice(s->grid->ctx->device);
    if (p->precision == DARE_PRECISION_FP64) return dare_bicgstab2_fp64_to(s, p, rep, f, field_written);
    return dare_bicgstab2_solve(s, p, rep);
}

int dare_bicgstab2_solve(dare_system* s, const dare_solver_params* p, dare_solve_report* rep) {
    if (!s || !p || !rep) return DARE_ERR_BAD_ARG;
    if (p->max_it < 0 || !(p->tol >= 0.)) return dare_gpu::set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "bicgstab2: bad params");
    if (p->precond != DARE_PREC_NONE && p->precond != DARE_PREC_JACOBI)
        return dare_gpu::set_error(s->grid->ctx, DARE_ERR_UNSUPPORTED, "bicgstab2: preconditioner not supported");
    cudaSetDevice(s->grid->ctx->device);
    if (p->precision == DARE_PRECISION_FP64) return dare_bicgstab2_fp64(s, p, rep);
    if (p->precision == DARE_PRECISION_FP32_REFINE) return dare_bicgstab2_refine(s, p, rep);
    return dare_gpu::set_error(s->grid->ctx, DARE_ERR_UNSUPPORTED, "bicgstab2: unknown precision mode");
}

}  // extern "C"
