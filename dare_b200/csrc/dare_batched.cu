// dare_batched.cu -- thousands of independent implicit diffusion steps of
// uneven sizes, each solved by Jacobi-BiCGStab(2), in one persistent launch.
//
// Every instance is a 3D box with constant D, one implicit-Euler step (DDT +
// div(D grad), DDT.inl:39-81, Divergence_Cartesian.inl:139-207) and
// Dirichlet / Neumann folding on its six faces (counter_diffusion1D.cpp:123-146).
// Its matrix is never stored: off-diagonals are one value per dimension and
// the diagonal depends only on which boundary faces a cell touches, so a
// 64-entry table per instance (indexed by that 6-bit mask) holds the
// assembled centre coefficient and its inverse, computed on the host with the
// same operation order as the assembly kernel.
//
// A persistent grid pulls instances from a device queue (heaviest first).
// One block solves one instance completely -- its reductions are block
// reductions, so there is no inter-block wait anywhere and results are
// deterministic -- and records the instance's own convergence status (the
// per-instance mask of the batch).  The block size and the cells each thread
// handles per sweep are tuned by dare_batch_autotune.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "dare_march.cuh"

using namespace dare_gpu;

namespace dare_gpu {

struct BInst {
    int n0, n1, n2, vec;
    int64_t off;          // first cell in the arena
    double tt;            // (V * 1) / dt
    double offd[3];       // off-diagonal per dimension: -(A_d * (dn_d * D))
    double tfold[6];      // rhs folding term 2 * bc * offd of each Dirichlet face (0 for Neumann)
    double C[64];         // centre coefficient per boundary mask
    double invd[64];      // 1 / C
};

struct BOut {
    int iters, converged, status, step;
    double res_abs, b_norm, tol_abs, pad;
};

struct BParams {
    double tol;
    int max_it;
    int tol_relative;
};

struct BVecs {
    double *x, *b, *rh, *r, *u, *v, *s, *w, *t;
};

}  // namespace dare_gpu

struct dare_batch {
    dare_ctx* ctx = nullptr;
    int device = 0;   // for dare_batch_destroy, which does not touch ctx
    int count = 0;
    int64_t total = 0;
    std::vector<dare_gpu::BInst> host;
    std::vector<int> order;          // solve order, heaviest first
    dare_gpu::BInst* d_inst = nullptr;
    int* d_order = nullptr;
    dare_gpu::BOut* d_out = nullptr;
    unsigned* d_queue = nullptr;
    double* arena = nullptr;         // 9 vectors of `total` cells
    int block = 512;
    int vec_by_size[8] = {1, 1, 1, 1, 1, 1, 1, 1};
};

namespace dare_gpu {

// the per-instance scalars a block keeps in registers
struct BGeom {
    int n0, n1, n2;
    double offd[3];
};

__device__ __forceinline__ int cell_mask(const BGeom& I, int i, int j, int k) {
    return (i == 0) | ((i == I.n0 - 1) << 1) | ((j == 0) << 2) | ((j == I.n1 - 1) << 3) | ((k == 0) << 4) |
           ((k == I.n2 - 1) << 5);
}

// block-wide sums of Q values, returned to every thread (fixed order)
template <int Q>
__device__ __forceinline__ void block_allsum(double (&v)[Q], double* sh) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) sh[q * 32 + wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) {
            double a = lane < nw ? sh[q * 32 + lane] : 0.;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
            if (lane == 0) sh[q * 32] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; q++) v[q] = sh[q * 32];
    __syncthreads();
}

// y = Ahat z at local cell c (Ahat = A D^-1: unit diagonal, off-diagonal
// offd_d * invd[mask(neighbour)]; neighbours past a face are absent)
__device__ __forceinline__ double ahat_row(const BGeom& I, const double* sinvd, const double* __restrict__ z,
                                           int c, int i, int j, int k) {
    const int p = I.n1 * I.n2;
    double y = z[c];
    if (i > 0) y += (I.offd[0] * sinvd[cell_mask(I, i - 1, j, k)]) * z[c - p];
    if (i < I.n0 - 1) y += (I.offd[0] * sinvd[cell_mask(I, i + 1, j, k)]) * z[c + p];
    if (j > 0) y += (I.offd[1] * sinvd[cell_mask(I, i, j - 1, k)]) * z[c - I.n2];
    if (j < I.n1 - 1) y += (I.offd[1] * sinvd[cell_mask(I, i, j + 1, k)]) * z[c + I.n2];
    if (k > 0) y += (I.offd[2] * sinvd[cell_mask(I, i, j, k - 1)]) * z[c - 1];
    if (k < I.n2 - 1) y += (I.offd[2] * sinvd[cell_mask(I, i, j, k + 1)]) * z[c + 1];
    return y;
}

// y = A z (unscaled, for the true residual)
__device__ __forceinline__ double a_row(const BGeom& I, const double* sC, const double* __restrict__ z, int c, int i,
                                        int j, int k) {
    const int p = I.n1 * I.n2;
    double y = sC[cell_mask(I, i, j, k)] * z[c];
    if (i > 0) y += I.offd[0] * z[c - p];
    if (i < I.n0 - 1) y += I.offd[0] * z[c + p];
    if (j > 0) y += I.offd[1] * z[c - I.n2];
    if (j < I.n1 - 1) y += I.offd[1] * z[c + I.n2];
    if (k > 0) y += I.offd[2] * z[c - 1];
    if (k < I.n2 - 1) y += I.offd[2] * z[c + 1];
    return y;
}

#define DARE_SWEEP(...)                                                           \
    for (int base_ = (int)threadIdx.x * vec; base_ < N; base_ += (int)blockDim.x * vec) { \
        for (int q_ = 0; q_ < vec; q_++) {                                        \
            const int c = base_ + q_;                                             \
            if (c >= N) break;                                                    \
            const int i = c / nyz, rem_ = c - i * nyz, j = rem_ / I.n2, k = rem_ - j * I.n2; \
            (void)i; (void)j; (void)k;                                            \
            __VA_ARGS__                                                           \
        }                                                                         \
    }

__global__ void __launch_bounds__(1024) k_batched(const BInst* __restrict__ insts, const int* __restrict__ order,
                                                  int count, BVecs vs, BParams prm, BOut* __restrict__ out,
                                                  unsigned* queue) {
    __shared__ double sh[32 * 5];
    __shared__ double sC[64], sinvd[64];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= count) break;
        const int id = order[item];
        const BInst* __restrict__ Ip = insts + id;
        if (threadIdx.x < 64) {
            sC[threadIdx.x] = Ip->C[threadIdx.x];
            sinvd[threadIdx.x] = Ip->invd[threadIdx.x];
        }
        __syncthreads();
        BGeom I;
        I.n0 = Ip->n0;
        I.n1 = Ip->n1;
        I.n2 = Ip->n2;
        I.offd[0] = Ip->offd[0];
        I.offd[1] = Ip->offd[1];
        I.offd[2] = Ip->offd[2];
        const double tt = Ip->tt;
        const int64_t off = Ip->off;
        const int N = I.n0 * I.n1 * I.n2, nyz = I.n1 * I.n2, vec = Ip->vec;
        double* __restrict__ x = vs.x + off;
        double* __restrict__ b = vs.b + off;
        double* __restrict__ rh = vs.rh + off;
        double* __restrict__ r = vs.r + off;
        double* __restrict__ u = vs.u + off;
        double* __restrict__ v = vs.v + off;
        double* __restrict__ s = vs.s + off;
        double* __restrict__ w = vs.w + off;
        double* __restrict__ t = vs.t + off;

        // Build: b = tt * phi_old then the Dirichlet folds (phi_old = x = the
        // initial guess, as the reference's Build copies the field into x)
        DARE_SWEEP({
            const int m = cell_mask(I, i, j, k);
            double rhs = 0. + tt * x[c];
            rhs += -1. * 0.;
#pragma unroll
            for (int f = 0; f < 6; f++)
                if (m & (1 << f)) rhs -= Ip->tfold[f];
            b[c] = rhs;
        })
        __syncthreads();
        // (0)-(2): r = b - Ahat y, r_hat_0 = r, u = v = w = 0
        double acc2[2] = {0., 0.};
        DARE_SWEEP({
            const double rr = b[c] - ahat_row(I, sinvd, x, c, i, j, k);
            r[c] = rr;
            rh[c] = rr;
            u[c] = 0.;
            v[c] = 0.;
            w[c] = 0.;
            acc2[0] += rr * rr;
            acc2[1] += b[c] * b[c];
        })
        block_allsum<2>(acc2, sh);
        const double bnorm = sqrt(acc2[1]);
        const double tol = prm.tol_relative ? prm.tol * bnorm : prm.tol;
        double rnorm = sqrt(acc2[0]);
        double alpha = 0., beta = 0., rho0 = 1., rho1 = 0., gamma = 0., omega2 = 1.;
        int k_it = 0, status = ST_RUNNING, step = 0;
        if (rnorm < tol) {
            status = ST_CONVERGED;
        } else if (isnan(rnorm)) {
            status = ST_NAN;
        } else {
            k_it = 1;
            rho1 = acc2[0];
        }
        bool tau0 = false;
        while (status == ST_RUNNING) {
            if (k_it > prm.max_it) {
                status = ST_MAXIT;
                break;
            }
            rho0 = -omega2 * rho0;                                     // (3)
            if (rho0 == 0.0) {
                status = ST_BREAKDOWN;
                step = 3;
                break;
            }
            beta = alpha * rho1 / rho0;                                // (4)
            rho0 = rho1;
            if (rho0 == 0.0) {
                status = ST_BREAKDOWN;
                step = 4;
                break;
            }
            DARE_SWEEP({ u[c] = r[c] - beta * u[c]; })                 // (5)
            __syncthreads();
            double a1[1] = {0.};
            DARE_SWEEP({                                               // (6), (7)
                const double vc = ahat_row(I, sinvd, u, c, i, j, k);
                v[c] = vc;
                a1[0] += vc * rh[c];
            })
            block_allsum<1>(a1, sh);
            gamma = a1[0];
            if (gamma == 0.0) {
                status = ST_BREAKDOWN;
                step = 7;
                break;
            }
            alpha = rho0 / gamma;
            DARE_SWEEP({                                               // (8), (10)
                r[c] = -alpha * v[c] + r[c];
                x[c] = alpha * u[c] + x[c];
            })
            __syncthreads();
            a1[0] = 0.;
            DARE_SWEEP({                                               // (9), (11)
                const double sc = ahat_row(I, sinvd, r, c, i, j, k);
                s[c] = sc;
                a1[0] += rh[c] * sc;
            })
            block_allsum<1>(a1, sh);
            rho1 = a1[0];
            beta = alpha * rho1 / rho0;
            rho0 = rho1;
            DARE_SWEEP({ v[c] = s[c] - beta * v[c]; })                 // (12)
            __syncthreads();
            a1[0] = 0.;
            DARE_SWEEP({                                               // (13), (14)
                const double wc = ahat_row(I, sinvd, v, c, i, j, k);
                w[c] = wc;
                a1[0] += wc * rh[c];
            })
            block_allsum<1>(a1, sh);
            gamma = a1[0];
            if (gamma == 0.0) {
                status = ST_BREAKDOWN;
                step = 14;
                break;
            }
            alpha = rho0 / gamma;
            DARE_SWEEP({                                               // (15)-(17)
                const double rc = r[c];
                u[c] = rc - beta * u[c];
                r[c] = -alpha * v[c] + rc;
                s[c] = -alpha * w[c] + s[c];
            })
            __syncthreads();
            double a5[5] = {0., 0., 0., 0., 0.};
            DARE_SWEEP({                                               // (18)-(20)
                const double tc = ahat_row(I, sinvd, s, c, i, j, k);
                t[c] = tc;
                const double rc = r[c], sc = s[c];
                a5[0] += rc * sc;
                a5[1] += sc * sc;
                a5[2] += sc * tc;
                a5[3] += tc * tc;
                a5[4] += rc * tc;
            })
            block_allsum<5>(a5, sh);
            double w1 = a5[0], mu = a5[1], nu = a5[2], tau = a5[3], w2 = a5[4];
            if (mu == 0.) {
                status = ST_BREAKDOWN;
                step = 20;
                break;
            }
            tau -= nu * nu / mu;                                       // (21)
            if (tau == 0.0) {
                tau0 = true;
                status = ST_BREAKDOWN;
                step = 21;
                break;
            }
            w2 = (w2 - (nu * w1) / mu) / tau;                          // (22)
            w1 = (w1 - nu * w2) / mu;                                  // (23)
            omega2 = w2;
            double a2[2] = {0., 0.};
            DARE_SWEEP({                                               // (24), (25), (25b)
                const double rc = r[c], sc = s[c];
                double xc = w1 * rc + w2 * sc + x[c];
                x[c] = alpha * u[c] + xc;
                const double rn = -w1 * sc + -w2 * t[c] + rc;
                r[c] = rn;
                u[c] = -w1 * v[c] + -w2 * w[c] + u[c];
                a2[0] += rn * rn;
                a2[1] += rh[c] * rn;
            })
            block_allsum<2>(a2, sh);
            rnorm = sqrt(a2[0]);
            if (rnorm <= tol && k_it > 1) {
                status = ST_CONVERGED;
                break;
            }
            if (isnan(rnorm)) {
                status = ST_NAN;
                break;
            }
            k_it += 1;
            rho1 = a2[1];
        }
        // x = M^-1 y
        DARE_SWEEP({ x[c] = sinvd[cell_mask(I, i, j, k)] * x[c]; })
        __syncthreads();
        bool converged = rnorm <= tol;
        if (tau0) {
            // BiCGStab2.inl:407-424: true residual; on failure M^-1 once more
            double a1[1] = {0.};
            DARE_SWEEP({
                const double rr = b[c] - a_row(I, sC, x, c, i, j, k);
                a1[0] += rr * rr;
            })
            block_allsum<1>(a1, sh);
            rnorm = sqrt(a1[0]);
            converged = rnorm <= tol;
            if (converged) {
                status = ST_CONVERGED;
                step = 0;
            } else {
                DARE_SWEEP({ x[c] = sinvd[cell_mask(I, i, j, k)] * x[c]; })
                __syncthreads();
            }
        }
        if (threadIdx.x == 0) {
            BOut o{};
            o.iters = k_it;
            o.converged = converged;
            o.status = status;
            o.step = step;
            o.res_abs = rnorm;
            o.b_norm = bnorm;
            o.tol_abs = tol;
            out[id] = o;
        }
        __syncthreads();
    }
}

#undef DARE_SWEEP

// size classes of the cells-per-thread table: <=16, <=24, <=32, <=48, <=64, <=96, <=128, larger
int size_class(int n) {
    static const int edges[7] = {16, 24, 32, 48, 64, 96, 128};
    int c = 0;
    while (c < 7 && n > edges[c]) c++;
    return c;
}

// Assembled coefficients of one instance, in the assembly kernel's order.
static int fill_instance(const dare_batch_instance& in, BInst& I) {
    for (int d = 0; d < 3; d++)
        if (in.n[d] < 3 || in.n[d] > 4096) return DARE_ERR_BAD_ARG;
    if (in.n[0] * in.n[1] * in.n[2] >= ((int64_t)1 << 31)) return DARE_ERR_BAD_ARG;
    for (int f = 0; f < 6; f++)
        if (in.bc_type[f] != DARE_BC_DIRICHLET && in.bc_type[f] != DARE_BC_NEUMANN) return DARE_ERR_BAD_ARG;
    if (!(in.dt > 0.) || !(in.D >= 0.)) return DARE_ERR_BAD_ARG;
    std::memset(&I, 0, sizeof(I));
    I.n0 = (int)in.n[0];
    I.n1 = (int)in.n[1];
    I.n2 = (int)in.n[2];
    I.vec = 1;
    double dx[3], V = 1., A[3], dn[3];
    for (int d = 0; d < 3; d++) dx[d] = in.size[d] / (double)in.n[d];     // CartesianMesh.inl:75-83
    for (int d = 0; d < 3; d++) V *= dx[d];
    for (int d = 0; d < 3; d++) A[d] = V / dx[d];
    for (int d = 0; d < 3; d++) dn[d] = 1. / dx[d];
    I.tt = (V * 1.) / in.dt;
    // diffusion face stencils and ApplyDivergence, then mb -= s
    double nb[7] = {0}, cf[7] = {0};
    for (int d = 0; d < 3; d++) {
        const int lo = 2 * d + 1, up = 2 * d + 2;
        nb[lo] = (-dn[d]) * in.D;
        cf[lo] = dn[d] * in.D;
        nb[up] = dn[d] * in.D;
        cf[up] = (-dn[d]) * in.D;
    }
    double sc[7] = {0};
    sc[DARE_EAST] = A[0] * nb[DARE_EAST];
    sc[DARE_CENTER] = A[0] * cf[DARE_EAST];
    sc[DARE_WEST] = -A[0] * nb[DARE_WEST];
    sc[DARE_CENTER] -= A[0] * cf[DARE_WEST];
    sc[DARE_NORTH] = A[1] * nb[DARE_NORTH];
    sc[DARE_CENTER] += A[1] * cf[DARE_NORTH];
    sc[DARE_SOUTH] = -A[1] * nb[DARE_SOUTH];
    sc[DARE_CENTER] -= A[1] * cf[DARE_SOUTH];
    sc[DARE_TOP] = A[2] * nb[DARE_TOP];
    sc[DARE_CENTER] += A[2] * cf[DARE_TOP];
    sc[DARE_BOTTOM] = -A[2] * nb[DARE_BOTTOM];
    sc[DARE_CENTER] -= A[2] * cf[DARE_BOTTOM];
    double coef[7];
    coef[DARE_CENTER] = I.tt;
    for (int p = 1; p < 7; p++) coef[p] = 0.;
    for (int p = 0; p < 7; p++) coef[p] += -1. * sc[p];
    for (int d = 0; d < 3; d++) I.offd[d] = coef[2 * d + 1];   // W == E, S == N, B == T
    for (int f = 0; f < 6; f++)
        I.tfold[f] = in.bc_type[f] == DARE_BC_DIRICHLET ? 2. * in.bc_value[f] * coef[f + 1] : 0.;
    for (int m = 0; m < 64; m++) {
        double C = coef[DARE_CENTER];
        for (int f = 0; f < 6; f++) {                               // fold W,E,S,N,B,T
            if (!(m & (1 << f))) continue;
            const double X = coef[f + 1];
            if (in.bc_type[f] == DARE_BC_DIRICHLET)
                C -= X;
            else
                C += X;
        }
        I.C[m] = C;
        I.invd[m] = 1. / C;
    }
    return DARE_OK;
}

static int launch_batch(dare_batch* bt, const dare_solver_params* p, int block) {
    dare_ctx* ctx = bt->ctx;
    BVecs vs;
    double* base = bt->arena;
    const int64_t T = bt->total;
    vs.x = base;
    vs.b = base + T;
    vs.rh = base + 2 * T;
    vs.r = base + 3 * T;
    vs.u = base + 4 * T;
    vs.v = base + 5 * T;
    vs.s = base + 6 * T;
    vs.w = base + 7 * T;
    vs.t = base + 8 * T;
    BParams prm{p->tol, p->max_it, p->tol_relative};
    DARE_CUDA(ctx, cudaMemsetAsync(bt->d_queue, 0, sizeof(unsigned), ctx->stream));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batched, block, 0);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * ctx->num_sms;
    if (blocks > bt->count) blocks = bt->count;
    k_batched<<<blocks, block, 0, ctx->stream>>>(bt->d_inst, bt->d_order, bt->count, vs, prm, bt->d_out,
                                                 bt->d_queue);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

static int upload_instances(dare_batch* bt) {
    dare_ctx* ctx = bt->ctx;
    for (auto& I : bt->host) {
        const int cls = size_class(std::max(I.n0, std::max(I.n1, I.n2)));
        I.vec = bt->vec_by_size[cls];
    }
    DARE_CUDA(ctx, cudaMemcpyAsync(bt->d_inst, bt->host.data(), sizeof(BInst) * bt->count, cudaMemcpyHostToDevice,
                                   ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

}  // namespace dare_gpu

extern "C" {

int dare_batch_create(dare_ctx* ctx, int count, const dare_batch_instance* inst, dare_batch** out) {
    using namespace dare_gpu;
    if (!ctx || !inst || !out || count < 1) return DARE_ERR_BAD_ARG;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    dare_batch* bt = new (std::nothrow) dare_batch();
    if (!bt) return DARE_ERR_OOM;
    bt->ctx = ctx;
    bt->device = ctx->device;
    bt->count = count;
    bt->host.resize(count);
    std::vector<double> work(count);
    int64_t off = 0;
    for (int q = 0; q < count; q++) {
        const int rc = fill_instance(inst[q], bt->host[q]);
        if (rc) {
            delete bt;
            return set_error(ctx, rc, "dare_batch_create: instance " + std::to_string(q) +
                                          " needs n >= 3 per dimension, Dirichlet/Neumann faces, dt > 0");
        }
        bt->host[q].off = off;
        const int64_t cells = (int64_t)bt->host[q].n0 * bt->host[q].n1 * bt->host[q].n2;
        off += (cells + 31) / 32 * 32;   // 256-byte aligned instances
        // expected work: cells x iteration estimate (diffusion number sigma = D dt / dx^2)
        const double dx = inst[q].size[0] / (double)inst[q].n[0];
        const double sigma = inst[q].D * inst[q].dt / (dx * dx);
        work[q] = (double)cells * (1. + std::sqrt(12. * sigma));
    }
    bt->total = off;
    bt->order.resize(count);
    for (int q = 0; q < count; q++) bt->order[q] = q;
    std::stable_sort(bt->order.begin(), bt->order.end(), [&](int a, int b) { return work[a] > work[b]; });
    cudaError_t e = cudaMalloc(&bt->d_inst, sizeof(BInst) * count);
    if (e == cudaSuccess) e = cudaMalloc(&bt->d_order, sizeof(int) * count);
    if (e == cudaSuccess) e = cudaMalloc(&bt->d_out, sizeof(BOut) * count);
    if (e == cudaSuccess) e = cudaMalloc(&bt->d_queue, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&bt->arena, sizeof(double) * 9 * (size_t)bt->total);
    if (e == cudaSuccess) e = cudaMemsetAsync(bt->arena, 0, sizeof(double) * (size_t)bt->total, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(bt->d_order, bt->order.data(), sizeof(int) * count, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        dare_batch_destroy(bt);
        return check_cuda(ctx, e, "dare_batch_create");
    }
    int rc = upload_instances(bt);
    if (rc) {
        dare_batch_destroy(bt);
        return rc;
    }
    *out = bt;
    return DARE_OK;
}

int dare_batch_destroy(dare_batch* bt) {
    if (!bt) return DARE_ERR_BAD_ARG;
    cudaSetDevice(bt->device);
    cudaFree(bt->d_inst);
    cudaFree(bt->d_order);
    cudaFree(bt->d_out);
    cudaFree(bt->d_queue);
    cudaFree(bt->arena);
    delete bt;
    return DARE_OK;
}

int64_t dare_batch_num_cells(const dare_batch* bt, int idx) {
    if (!bt || idx < 0 || idx >= bt->count) return -1;
    const auto& I = bt->host[idx];
    return (int64_t)I.n0 * I.n1 * I.n2;
}

int dare_batch_set_field(dare_batch* bt, int idx, const double* host_phi) {
    if (!bt || !host_phi || idx < 0 || idx >= bt->count) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = bt->ctx;
    const auto& I = bt->host[idx];
    DARE_CUDA(ctx, cudaMemcpyAsync(bt->arena + I.off, host_phi, sizeof(double) * (size_t)I.n0 * I.n1 * I.n2,
                                   cudaMemcpyHostToDevice, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_batch_get_field(dare_batch* bt, int idx, double* host_phi) {
    if (!bt || !host_phi || idx < 0 || idx >= bt->count) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = bt->ctx;
    const auto& I = bt->host[idx];
    DARE_CUDA(ctx, cudaMemcpyAsync(host_phi, bt->arena + I.off, sizeof(double) * (size_t)I.n0 * I.n1 * I.n2,
                                   cudaMemcpyDeviceToHost, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_batch_zero_fields(dare_batch* bt) {
    if (!bt) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = bt->ctx;
    cudaSetDevice(ctx->device);
    DARE_CUDA(ctx, cudaMemsetAsync(bt->arena, 0, sizeof(double) * (size_t)bt->total, ctx->stream));
    return DARE_OK;
}

int dare_batch_solve(dare_batch* bt, const dare_solver_params* p, dare_batch_report* reports) {
    using namespace dare_gpu;
    if (!bt || !p) return DARE_ERR_BAD_ARG;
    if (p->precond != DARE_PREC_JACOBI || p->precision != DARE_PRECISION_FP64)
        return set_error(bt->ctx, DARE_ERR_UNSUPPORTED, "dare_batch_solve: FP64 Jacobi-BiCGStab2 only");
    dare_ctx* ctx = bt->ctx;
    cudaSetDevice(ctx->device);
    int rc = launch_batch(bt, p, bt->block);
    if (rc) return rc;
    if (reports) {
        std::vector<BOut> o(bt->count);
        DARE_CUDA(ctx, cudaMemcpyAsync(o.data(), bt->d_out, sizeof(BOut) * bt->count, cudaMemcpyDeviceToHost,
                                       ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (int q = 0; q < bt->count; q++) {
            dare_batch_report& r = reports[q];
            r.iters = o[q].iters;
            r.converged = o[q].converged;
            r.status = o[q].status == ST_CONVERGED ? DARE_SOLVE_CONVERGED
                       : o[q].status == ST_MAXIT  ? DARE_SOLVE_MAXIT
                       : o[q].status == ST_NAN    ? DARE_SOLVE_NAN
                                                  : DARE_SOLVE_BREAKDOWN;
            r.breakdown_step = o[q].step;
            r.res_abs = o[q].res_abs;
            r.b_norm = o[q].b_norm;
            r.tol_abs = o[q].tol_abs;
        }
    }
    return DARE_OK;
}

// Tunes (1) cells per thread per sweep for each size class, from single-class
// sub-batches, and (2) the block size for the whole batch, by timing solves
// of copies of the current fields (restored afterwards).
int dare_batch_autotune(dare_batch* bt, const dare_solver_params* p, int* chosen_block) {
    using namespace dare_gpu;
    if (!bt || !p) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = bt->ctx;
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(double) * (size_t)bt->total;
    double* saved = nullptr;
    DARE_CUDA(ctx, cudaMalloc(&saved, bytes));
    DARE_CUDA(ctx, cudaMemcpyAsync(saved, bt->arena, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](int block) -> double {
        cudaMemcpyAsync(bt->arena, saved, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
        cudaEventRecord(e0, ctx->stream);
        if (launch_batch(bt, p, block)) return 1e30;
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    static const int blocks[3] = {256, 512, 1024};
    static const int vecs[3] = {1, 2, 4};
    int best_block = bt->block;
    double best_t = 1e30;
    for (int bi = 0; bi < 3; bi++) {
        // per size class: pick cells per thread with all instances at that setting
        for (int vi = 0; vi < 3; vi++) {
            for (int c = 0; c < 8; c++) bt->vec_by_size[c] = vecs[vi];
            if (upload_instances(bt)) break;
            const double tm = timed(blocks[bi]);
            if (tm < best_t) {
                best_t = tm;
                best_block = blocks[bi];
                for (int c = 0; c < 8; c++) bt->vec_by_size[c] = vecs[vi];
            }
        }
    }
    // keep the best uniform setting, then refine each size class separately
    int base_vec = bt->vec_by_size[0];
    for (int c = 0; c < 8; c++) bt->vec_by_size[c] = base_vec;
    for (int c = 0; c < 8; c++) {
        bool present = false;
        for (const auto& I : bt->host)
            if (size_class(std::max(I.n0, std::max(I.n1, I.n2))) == c) present = true;
        if (!present) continue;
        int best_v = base_vec;
        for (int vi = 0; vi < 3; vi++) {
            if (vecs[vi] == base_vec) continue;
            bt->vec_by_size[c] = vecs[vi];
            if (upload_instances(bt)) break;
            const double tm = timed(best_block);
            if (tm < best_t) {
                best_t = tm;
                best_v = vecs[vi];
            }
        }
        bt->vec_by_size[c] = best_v;
    }
    int rc = upload_instances(bt);
    bt->block = best_block;
    cudaMemcpyAsync(bt->arena, saved, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(saved);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (chosen_block) *chosen_block = best_block;
    return rc;
}

int dare_batch_get_tuning(const dare_batch* bt, int* block, int vec_by_size[8]) {
    if (!bt) return DARE_ERR_BAD_ARG;
    if (block) *block = bt->block;
    if (vec_by_size)
        for (int c = 0; c < 8; c++) vec_by_size[c] = bt->vec_by_size[c];
    return DARE_OK;
}

}  // extern "C"
