// dare_bicgstab2.cu -- device-resident BiCGStab(2) for the structured
// 7-point systems (MatrixSystem/BiCGStab2.inl:166-582, van der Vorst's
// unrolled Sleijpen-Fokkema form, right preconditioner).
//
// Design (HBM-bound; every kernel streams its operands once):
//   * Jacobi is folded into the operator: Ahat = A D^-1 (column scaling), so
//     Ahat has a unit diagonal and each SpMV reads 6 off-diagonals.  The
//     iteration runs in the preconditioned variable y (x = D^-1 y), exactly
//     as the reference: r0 = b - A M^-1 x_init, x = M^-1 y at the end.
//   * One iteration = 5 kernels.  Each fuses the axpy that produces its SpMV
//     input (evaluated at the 7 stencil points from the two source vectors,
//     the result written once at the centre) with the SpMV and the dot
//     products that follow it.  Vectors written that way are double
//     buffered (u and r flip every iteration, v and s have a fixed pair), so
//     a graph captures two iterations.
//   * Scalars (alpha, beta, rho, omega, ...) never leave the device: the last
//     block of each kernel reduces the per-block partials in a fixed order
//     (deterministic, no floating-point atomics), evaluates the reference's
//     scalar recurrence and its breakdown checks, and sets a done flag that
//     turns every later kernel into a no-op.  The host polls that flag every
//     few iterations.
//   * The reference keeps omega/mu/nu/tau in long double; here they are FP64.
#include <cmath>
#include <cstring>
#include <new>

#include "dare_internal.cuh"

using namespace dare_gpu;

namespace dare_gpu {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;
constexpr int kMaxQ = 5;

enum : int { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXIT = 2, ST_BREAKDOWN = 3, ST_NAN = 4, ST_TAU0 = 5 };

struct SolverState {
    double alpha, beta, rho0, rho1, gamma, omega1, omega2, mu, nu, tau;
    double rnorm, rnorm0, bnorm2, tol;
    int k, max_it, done, status, step, tol_relative;
    unsigned int count;
};

struct Op {
    const double* __restrict__ c;    // centre diagonal (general operator only)
    const double* __restrict__ off;  // 6 off-diagonal arrays W,E,S,N,B,T, each n long
    int64_t n;
};

struct Vecs {
    double* x;        // y in the preconditioned variable, x at the end
    const double* b;
    double* rh;       // r_hat_0
    double* r[2];
    double* u[2];
    double* v[2];
    double* s[2];
    double* w;
    double* t;
};

}  // namespace dare_gpu

struct dare_solver_ws {
    int64_t n = 0;
    double* ahat = nullptr;      // 6 * n
    double* invd = nullptr;      // n
    double* vec = nullptr;       // 12 * n work vectors
    double* partials = nullptr;  // kMaxQ * kMaxBlocks
    SolverState* st = nullptr;
    SolverState* st_host = nullptr;  // pinned
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [jacobi?][profiling?]
    int graph_blocks = 0;
};

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
    delete ws;
}

namespace dare_gpu {

// ---------------------------------------------------------------------------
// cell helpers
// ---------------------------------------------------------------------------
struct CellIdx {
    int i, j, k;
};

__device__ __forceinline__ CellIdx split(const GridDev& g, int64_t c) {
    const unsigned nz = (unsigned)g.n[2], ny = (unsigned)g.n[1];
    const unsigned cc = (unsigned)c;
    const unsigned row = cc / nz;
    CellIdx r;
    r.k = (int)(cc - row * nz);
    r.i = (int)(row / ny);
    r.j = (int)(row - (unsigned)r.i * ny);
    return r;
}

template <bool UNIT>
__device__ __forceinline__ double apply_row(const Op& op, int64_t c, const double z[7]) {
    const int64_t n = op.n;
    double y = UNIT ? z[0] : op.c[c] * z[0];
    y += op.off[c] * z[1];
    y += op.off[n + c] * z[2];
    y += op.off[2 * n + c] * z[3];
    y += op.off[3 * n + c] * z[4];
    y += op.off[4 * n + c] * z[5];
    y += op.off[5 * n + c] * z[6];
    return y;
}

// Block reduction of Q values; thread 0 gets the sums. Fixed order.
template <int Q>
__device__ __forceinline__ void block_sum(double (&v)[Q], double* sh /* [32*Q] */) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) sh[q * 32 + wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < Q; q++) {
            double a = lane < nw ? sh[q * 32 + lane] : 0.;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
            v[q] = a;
        }
    }
}

// Publish this block's partial sums; returns true in the last block to
// finish, after which tot[] holds the grid-wide sums (fixed summation order).
template <int Q>
__device__ bool grid_reduce(double (&v)[Q], double* __restrict__ partials, unsigned int* counter,
                            double (&tot)[Q]) {
    __shared__ double sh[32 * kMaxQ];
    __shared__ bool is_last;
    block_sum<Q>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) partials[q * kMaxBlocks + blockIdx.x] = v[q];
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double a[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) a[q] = 0.;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < Q; q++) a[q] += __ldcg(partials + q * kMaxBlocks + b);
    }
    __syncthreads();
    block_sum<Q>(a, sh);
#pragma unroll
    for (int q = 0; q < Q; q++) tot[q] = a[q];
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

__device__ __forceinline__ void finish(SolverState* st, int status, int step) {
    st->status = status;
    st->step = step;
    st->done = 1;
}

// Loop-top bookkeeping of the reference: `if (k > max_iteration) break;`,
// step (3) and step (4) given rho1 = <r_hat_0, r>.
__device__ void begin_iteration(SolverState* st, double rho1) {
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

// ---------------------------------------------------------------------------
// set-up kernels
// ---------------------------------------------------------------------------
__global__ void k_invdiag(const double* __restrict__ dc, double* __restrict__ invd, int64_t n) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        invd[c] = 1. / dc[c];
}

// Ahat[p][c] = A[p][c] * invd[neighbour_p(c)]  (right Jacobi folded in)
__global__ void k_fold_jacobi(GridDev g, const double* __restrict__ diag, const double* __restrict__ invd,
                              double* __restrict__ ahat) {
    const int64_t n = g.ncell;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
#pragma unroll
        for (int p = 1; p < 7; p++) ahat[(p - 1) * n + c] = diag[p * n + c] * invd[nb[p]];
    }
}

// K0: r = b - Op x; r_hat_0 = r; u = v = w = 0; sums <r,r>, <b,b>.
template <bool UNIT>
__global__ void __launch_bounds__(kThreads) k_init(GridDev g, Op op, Vecs vs, SolverState* st,
                                                   double* partials) {
    const int64_t n = g.ncell;
    double acc[2] = {0., 0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
        double z[7];
#pragma unroll
        for (int p = 0; p < 7; p++) z[p] = vs.x[nb[p]];
        const double bc = vs.b[c];
        const double r = bc - apply_row<UNIT>(op, c, z);   // r.update(-1, v, 1)
        vs.r[0][c] = r;
        vs.rh[c] = r;
        vs.u[0][c] = 0.;
        vs.v[0][c] = 0.;
        vs.w[c] = 0.;
        acc[0] += r * r;
        acc[1] += bc * bc;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        st->bnorm2 = tot[1];
        if (st->tol_relative) st->tol = st->tol * sqrt(tot[1]);
        st->rnorm0 = sqrt(tot[0]);
        st->rnorm = st->rnorm0;
        st->alpha = 0.;                                       // BiCGStab2.inl:182
        st->rho0 = st->omega1 = st->omega2 = 1.;             // (1)
        st->k = 0;
        if (st->rnorm0 < st->tol) {                           // initial guess converged
            finish(st, ST_CONVERGED, 0);
            return;
        }
        if (isnan(st->rnorm0)) {
            finish(st, ST_NAN, 0);
            return;
        }
        st->k = 1;
        begin_iteration(st, tot[0]);                          // <r_hat_0, r> = <r, r>
    }
}

// K1: (5) u = r - beta u; (6) v = Op u; (7) gamma = <v, r_hat_0>, alpha = rho0/gamma
template <bool UNIT>
__global__ void __launch_bounds__(kThreads) k_step1(GridDev g, Op op, const double* __restrict__ r,
                                                    const double* __restrict__ u_in, double* __restrict__ u_out,
                                                    double* __restrict__ v, const double* __restrict__ rh,
                                                    SolverState* st, double* partials) {
    if (st->done) return;
    const double beta = st->beta;
    const int64_t n = g.ncell;
    double acc[1] = {0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
        double z[7];
#pragma unroll
        for (int p = 0; p < 7; p++) z[p] = r[nb[p]] - beta * u_in[nb[p]];
        u_out[c] = z[0];
        const double vc = apply_row<UNIT>(op, c, z);
        v[c] = vc;
        acc[0] += vc * rh[c];
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        st->gamma = tot[0];
        if (st->gamma == 0.0) {
            finish(st, ST_BREAKDOWN, 7);
            return;
        }
        st->alpha = st->rho0 / st->gamma;
    }
}

// K2: (8) r = r - alpha v; (9) s = Op r; (10) x = x + alpha u;
//     (11) rho1 = <r_hat_0, s>, beta = alpha rho1 / rho0, rho0 = rho1
template <bool UNIT>
__global__ void __launch_bounds__(kThreads) k_step2(GridDev g, Op op, const double* __restrict__ r_in,
                                                    double* __restrict__ r_out, const double* __restrict__ v,
                                                    double* __restrict__ s, double* __restrict__ x,
                                                    const double* __restrict__ u, const double* __restrict__ rh,
                                                    SolverState* st, double* partials) {
    if (st->done) return;
    const double alpha = st->alpha;
    const int64_t n = g.ncell;
    double acc[1] = {0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
        double z[7];
#pragma unroll
        for (int p = 0; p < 7; p++) z[p] = -alpha * v[nb[p]] + r_in[nb[p]];
        r_out[c] = z[0];
        const double sc = apply_row<UNIT>(op, c, z);
        s[c] = sc;
        x[c] = alpha * u[c] + x[c];
        acc[0] += rh[c] * sc;
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        st->rho1 = tot[0];
        st->beta = st->alpha * st->rho1 / st->rho0;
        st->rho0 = st->rho1;
    }
}

// K3: (12) v = s - beta v; (13) w = Op v; (14) gamma = <w, r_hat_0>, alpha = rho0/gamma
template <bool UNIT>
__global__ void __launch_bounds__(kThreads) k_step3(GridDev g, Op op, const double* __restrict__ s,
                                                    const double* __restrict__ v_in, double* __restrict__ v_out,
                                                    double* __restrict__ w, const double* __restrict__ rh,
                                                    SolverState* st, double* partials) {
    if (st->done) return;
    const double beta = st->beta;
    const int64_t n = g.ncell;
    double acc[1] = {0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
        double z[7];
#pragma unroll
        for (int p = 0; p < 7; p++) z[p] = s[nb[p]] - beta * v_in[nb[p]];
        v_out[c] = z[0];
        const double wc = apply_row<UNIT>(op, c, z);
        w[c] = wc;
        acc[0] += wc * rh[c];
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        st->gamma = tot[0];
        if (st->gamma == 0.0) {
            finish(st, ST_BREAKDOWN, 14);
            return;
        }
        st->alpha = st->rho0 / st->gamma;
    }
}

// K4: (15) u = r - beta u; (16) r = r - alpha v; (17) s = s - alpha w; (18) t = Op s;
//     (19)-(20) <r,s>, <s,s>, <s,t>, <t,t>, <r,t>; (21)-(23) omega
template <bool UNIT>
__global__ void __launch_bounds__(kThreads) k_step4(GridDev g, Op op, double* __restrict__ u,
                                                    double* __restrict__ r, const double* __restrict__ v,
                                                    const double* __restrict__ s_in, double* __restrict__ s_out,
                                                    const double* __restrict__ w, double* __restrict__ t,
                                                    SolverState* st, double* partials) {
    if (st->done) return;
    const double alpha = st->alpha, beta = st->beta;
    const int64_t n = g.ncell;
    double acc[5] = {0., 0., 0., 0., 0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
        const double rc = r[c];
        u[c] = rc - beta * u[c];                              // (15)
        const double rn = -alpha * v[c] + rc;                 // (16)
        r[c] = rn;
        double z[7];
#pragma unroll
        for (int p = 0; p < 7; p++) z[p] = -alpha * w[nb[p]] + s_in[nb[p]];   // (17)
        s_out[c] = z[0];
        const double tc = apply_row<UNIT>(op, c, z);          // (18)
        t[c] = tc;
        acc[0] += rn * z[0];
        acc[1] += z[0] * z[0];
        acc[2] += z[0] * tc;
        acc[3] += tc * tc;
        acc[4] += rn * tc;
    }
    double tot[5];
    if (!grid_reduce<5>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
        double omega_1 = tot[0], mu = tot[1], nu = tot[2], tau = tot[3], omega_2 = tot[4];
        if (mu == 0.) {
            finish(st, ST_BREAKDOWN, 20);
            return;
        }
        tau -= nu * nu / mu;                                  // (21)
        st->mu = mu;
        st->nu = nu;
        st->tau = tau;
        if (tau == 0.0) {
            finish(st, ST_TAU0, 21);
            return;
        }
        omega_2 = (omega_2 - (nu * omega_1) / mu) / tau;      // (22)
        omega_1 = (omega_1 - nu * omega_2) / mu;              // (23)
        st->omega1 = omega_1;
        st->omega2 = omega_2;
    }
}

// K5: (24) x = x + w1 r + w2 s + alpha u; (25) r = r - w1 s - w2 t; ||r||;
//     u = u - w1 v - w2 w; then the next iteration's (3), (4).
__global__ void __launch_bounds__(kThreads) k_step5(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                    const double* __restrict__ s, const double* __restrict__ t,
                                                    double* __restrict__ u, const double* __restrict__ v,
                                                    const double* __restrict__ w, const double* __restrict__ rh,
                                                    SolverState* st, double* partials) {
    if (st->done) return;
    const double w1 = st->omega1, w2 = st->omega2, alpha = st->alpha;
    double acc[2] = {0., 0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const double rc = r[c], sc = s[c];
        double xc = w1 * rc + w2 * sc + x[c];
        xc = alpha * u[c] + xc;
        x[c] = xc;
        const double rn = -w1 * sc + -w2 * t[c] + rc;
        r[c] = rn;
        u[c] = -w1 * v[c] + -w2 * w[c] + u[c];
        acc[0] += rn * rn;
        acc[1] += rh[c] * rn;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) {
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
}

// x = invd .* x (applyRightPrec at the end of the solve)
__global__ void k_scale(int64_t n, const double* __restrict__ invd, double* __restrict__ x) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        x[c] = invd[c] * x[c];
}

// ||b - A x||^2 with the assembled (unscaled) operator, FP64
__global__ void __launch_bounds__(kThreads) k_true_residual(GridDev g, Op op, const double* __restrict__ x,
                                                            const double* __restrict__ b, SolverState* st,
                                                            double* partials, double* out) {
    const int64_t n = g.ncell;
    double acc[1] = {0.};
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const CellIdx ci = split(g, c);
        int64_t nb[7];
        neighbour_ordinals(g, ci.i, ci.j, ci.k, c, nb);
        double z[7];
#pragma unroll
        for (int p = 0; p < 7; p++) z[p] = x[nb[p]];
        const double r = b[c] - apply_row<false>(op, c, z);
        acc[0] += r * r;
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &st->count, tot)) return;
    if (threadIdx.x == 0) *out = sqrt(tot[0]);
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct Launch {
    int blocks;
};

static int ensure_ws(dare_system* s) {
    dare_ctx* ctx = s->grid->ctx;
    const int64_t n = s->grid->dev.ncell;
    if (s->ws && s->ws->n == n) return DARE_OK;
    dare_solver_ws_free(s->ws);
    s->ws = nullptr;
    dare_solver_ws* ws = new (std::nothrow) dare_solver_ws();
    if (!ws) return DARE_ERR_OOM;
    ws->n = n;
    cudaError_t e = cudaMalloc(&ws->ahat, (size_t)n * 6 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->invd, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->vec, (size_t)n * 12 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->partials, (size_t)kMaxQ * kMaxBlocks * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ws->st, sizeof(SolverState));
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->st, 0, sizeof(SolverState), ctx->stream);
    if (e == cudaSuccess) e = cudaMallocHost(&ws->st_host, sizeof(SolverState));
    if (e != cudaSuccess) {
        dare_solver_ws_free(ws);
        return check_cuda(ctx, e, "bicgstab2 workspace");
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step4<true>, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    ws->graph_blocks = grid_blocks(ctx, n, kThreads, per_sm);
    if (ws->graph_blocks > kMaxBlocks) ws->graph_blocks = kMaxBlocks;
    s->ws = ws;
    return DARE_OK;
}

static Vecs make_vecs(dare_system* s) {
    dare_solver_ws* ws = s->ws;
    const int64_t n = ws->n;
    Vecs v;
    v.x = s->x;
    v.b = s->rhs;
    double* base = ws->vec;
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

// Launch one iteration; `par` selects which halves of r/u are current.
// `ev` (optional, profiling): ev[0] is recorded before the first kernel,
// ev[1..5] after each of the five kernels.
template <bool UNIT>
static int launch_iteration(dare_ctx* ctx, const GridDev& g, const Op& op, const Vecs& vs, SolverState* st,
                            double* partials, int blocks, int par, cudaEvent_t* ev) {
    const int a = par, b = 1 - par;
    cudaStream_t sm = ctx->stream;
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[0], sm));
    k_step1<UNIT><<<blocks, kThreads, 0, sm>>>(g, op, vs.r[a], vs.u[a], vs.u[b], vs.v[0], vs.rh, st, partials);
    DARE_LAUNCHED(ctx);
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[1], sm));
    k_step2<UNIT><<<blocks, kThreads, 0, sm>>>(g, op, vs.r[a], vs.r[b], vs.v[0], vs.s[0], vs.x, vs.u[b], vs.rh, st,
                                              partials);
    DARE_LAUNCHED(ctx);
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[2], sm));
    k_step3<UNIT><<<blocks, kThreads, 0, sm>>>(g, op, vs.s[0], vs.v[0], vs.v[1], vs.w, vs.rh, st, partials);
    DARE_LAUNCHED(ctx);
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[3], sm));
    k_step4<UNIT><<<blocks, kThreads, 0, sm>>>(g, op, vs.u[b], vs.r[b], vs.v[1], vs.s[0], vs.s[1], vs.w, vs.t, st,
                                              partials);
    DARE_LAUNCHED(ctx);
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[4], sm));
    k_step5<<<blocks, kThreads, 0, sm>>>(g.ncell, vs.x, vs.r[b], vs.s[1], vs.t, vs.u[b], vs.v[1], vs.w, vs.rh, st,
                                         partials);
    DARE_LAUNCHED(ctx);
    if (ev) DARE_CUDA(ctx, cudaEventRecord(ev[5], sm));
    return DARE_OK;
}

template <bool UNIT>
static int build_graph(dare_system* s, const Op& op, cudaGraphExec_t* out, bool profile) {
    dare_ctx* ctx = s->grid->ctx;
    dare_solver_ws* ws = s->ws;
    Vecs vs = make_vecs(s);
    cudaStream_t cap;
    DARE_CUDA(ctx, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaStream_t saved = ctx->stream;
    ctx->stream = cap;
    cudaGraph_t graph = nullptr;
    int rc = DARE_OK;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = launch_iteration<UNIT>(ctx, s->grid->dev, op, vs, ws->st, ws->partials, ws->graph_blocks, 0,
                                    profile ? ctx->ev : nullptr);
        if (rc == DARE_OK)
            rc = launch_iteration<UNIT>(ctx, s->grid->dev, op, vs, ws->st, ws->partials, ws->graph_blocks, 1,
                                        profile ? ctx->ev + 5 : nullptr);
        cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
        if (e == cudaSuccess) e = e2;
    }
    ctx->stream = saved;
    ctx->launches -= 10;  // captured, not executed
    if (e == cudaSuccess && rc == DARE_OK) e = cudaGraphInstantiate(out, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != DARE_OK) return rc;
    if (e != cudaSuccess) return check_cuda(ctx, e, "bicgstab2 graph capture");
    return DARE_OK;
}

}  // namespace dare_gpu

// Shared by the FP64 solve and the refinement driver.
int dare_bicgstab2_fp64(dare_system* s, const dare_solver_params* p, dare_solve_report* rep) {
    using namespace dare_gpu;
    dare_ctx* ctx = s->grid->ctx;
    const GridDev& g = s->grid->dev;
    int rc = ensure_ws(s);
    if (rc) return rc;
    dare_solver_ws* ws = s->ws;
    const int64_t n = g.ncell;
    const bool jacobi = p->precond == DARE_PREC_JACOBI;
    const int blocks = ws->graph_blocks;
    const int eb = grid_blocks(ctx, n, 256, 8);

    Op full{s->diag, s->diag + n, n};
    Op folded{nullptr, ws->ahat, n};
    if (jacobi) {
        k_invdiag<<<eb, 256, 0, ctx->stream>>>(s->diag, ws->invd, n);
        DARE_LAUNCHED(ctx);
        k_fold_jacobi<<<eb, 256, 0, ctx->stream>>>(g, s->diag, ws->invd, ws->ahat);
        DARE_LAUNCHED(ctx);
    }
    SolverState init{};
    init.tol = p->tol;
    init.max_it = p->max_it;
    init.tol_relative = p->tol_relative;
    DARE_CUDA(ctx, cudaMemcpyAsync(ws->st, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    Vecs vs = make_vecs(s);
    if (jacobi)
        k_init<true><<<blocks, kThreads, 0, ctx->stream>>>(g, folded, vs, ws->st, ws->partials);
    else
        k_init<false><<<blocks, kThreads, 0, ctx->stream>>>(g, full, vs, ws->st, ws->partials);
    DARE_LAUNCHED(ctx);

    const bool prof = ctx->profiling != 0;
    cudaGraphExec_t& ge = ws->graph[jacobi ? 1 : 0][prof ? 1 : 0];
    if (!ge) {
        rc = jacobi ? build_graph<true>(s, folded, &ge, prof) : build_graph<false>(s, full, &ge, prof);
        if (rc) return rc;
    }
    int check_every = p->check_every;
    if (check_every <= 0) {
        const int64_t per = (int64_t)1 << 21;
        check_every = (int)((per + n - 1) / n);
        if (check_every < 1) check_every = 1;
        if (check_every > 8) check_every = 8;
    }
    const int max_graphs = p->max_it / 2 + 2;
    for (int gi = 0; gi < max_graphs; gi++) {
        DARE_CUDA(ctx, cudaGraphLaunch(ge, ctx->stream));
        ctx->launches += 10;
        if ((gi + 1) % check_every == 0 || gi + 1 == max_graphs) {
            DARE_CUDA(ctx, cudaMemcpyAsync(ws->st_host, ws->st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx->stream));
            DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (ws->st_host->done) break;
            if (prof && check_every == 1) {
                // all ten kernels of this graph did real work: record their durations
                for (int it = 0; it < 2; it++)
                    for (int q = 0; q < 5; q++) {
                        float ms = 0.f;
                        if (cudaEventElapsedTime(&ms, ctx->ev[it * 5 + q], ctx->ev[it * 5 + q + 1]) == cudaSuccess) {
                            ctx->stat_ms[KID_STEP1 + q] += ms;
                            ctx->stat_n[KID_STEP1 + q] += 1;
                        }
                    }
            }
        }
    }
    DARE_CUDA(ctx, cudaMemcpyAsync(ws->st_host, ws->st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    SolverState st = *ws->st_host;
    if (!st.done) return set_error(ctx, DARE_ERR_STATE, "bicgstab2: iteration bound reached without a status");

    std::memset(rep, 0, sizeof(*rep));
    rep->iters = st.k;
    rep->b_norm = sqrt(st.bnorm2);
    rep->res_abs = st.rnorm;
    rep->breakdown_step = st.step;
    rep->tol_abs = st.tol;
    double* dres = ws->partials + (kMaxQ - 1) * kMaxBlocks + kMaxBlocks - 1;  // scratch slot
    if (st.status == ST_TAU0) {
        // BiCGStab2.inl:407-424: x = M^-1 y, true residual, return if converged;
        // otherwise break to the common exit, which applies M^-1 once more.
        if (jacobi) {
            k_scale<<<eb, 256, 0, ctx->stream>>>(n, ws->invd, s->x);
            DARE_LAUNCHED(ctx);
        }
        k_true_residual<<<blocks, kThreads, 0, ctx->stream>>>(g, full, s->x, s->rhs, ws->st, ws->partials, dres);
        DARE_LAUNCHED(ctx);
        double tr = 0.;
        DARE_CUDA(ctx, cudaMemcpyAsync(&tr, dres, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        rep->res_abs = tr;
        if (tr <= st.tol) {
            rep->converged = 1;
            rep->status = DARE_SOLVE_CONVERGED;
            rep->breakdown_step = 0;
        } else {
            if (jacobi) {
                k_scale<<<eb, 256, 0, ctx->stream>>>(n, ws->invd, s->x);
                DARE_LAUNCHED(ctx);
            }
            rep->converged = 0;
            rep->status = DARE_SOLVE_BREAKDOWN;
        }
    } else {
        if (jacobi) {
            k_scale<<<eb, 256, 0, ctx->stream>>>(n, ws->invd, s->x);
            DARE_LAUNCHED(ctx);
        }
        rep->converged = st.rnorm <= st.tol;
        switch (st.status) {
        case ST_CONVERGED: rep->status = DARE_SOLVE_CONVERGED; break;
        case ST_MAXIT: rep->status = DARE_SOLVE_MAXIT; break;
        case ST_NAN: rep->status = DARE_SOLVE_NAN; break;
        default: rep->status = DARE_SOLVE_BREAKDOWN; break;
        }
    }
    if (p->compute_true_residual) {
        k_true_residual<<<blocks, kThreads, 0, ctx->stream>>>(g, full, s->x, s->rhs, ws->st, ws->partials, dres);
        DARE_LAUNCHED(ctx);
        double tr = 0.;
        DARE_CUDA(ctx, cudaMemcpyAsync(&tr, dres, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        rep->true_res_abs = tr;
    }
    return DARE_OK;
}

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

int dare_bicgstab2_solve(dare_system* s, const dare_solver_params* p, dare_solve_report* rep) {
    if (!s || !p || !rep) return DARE_ERR_BAD_ARG;
    if (p->max_it < 0 || !(p->tol >= 0.)) return dare_gpu::set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "bicgstab2: bad params");
    if (p->precond != DARE_PREC_NONE && p->precond != DARE_PREC_JACOBI)
        return dare_gpu::set_error(s->grid->ctx, DARE_ERR_UNSUPPORTED, "bicgstab2: preconditioner not supported");
    cudaSetDevice(s->grid->ctx->device);
    if (p->precision == DARE_PRECISION_FP64) return dare_bicgstab2_fp64(s, p, rep);
    return dare_gpu::set_error(s->grid->ctx, DARE_ERR_UNSUPPORTED, "bicgstab2: precision mode not built");
}

}  // extern "C"
