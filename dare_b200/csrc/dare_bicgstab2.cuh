// dare_bicgstab2.cuh -- solver types shared by the FP64 solve, the
// FP32-inner / FP64-refinement driver and the batched solver.
#pragma once

#include "dare_internal.cuh"

namespace dare_gpu {

constexpr int kMaxBlocks = 16384;   // per-block partial slots of one reduction
constexpr int kMaxQ = 5;            // dot products fused into one kernel

enum : int { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXIT = 2, ST_BREAKDOWN = 3, ST_NAN = 4, ST_TAU0 = 5 };

struct SolverState {
    double alpha, beta, rho0, rho1, gamma, omega1, omega2, mu, nu, tau;
    double rnorm, rnorm0, bnorm2, tol;
    double alpha1, beta1;  // learned solve: alpha of step 7 and beta of step 11 (its flexible update)
    int k, max_it, done, status, step, tol_relative;
    unsigned int count;   // reduction arrivals (reset by the last arrival)
    unsigned int queue;   // next work item of a marching kernel
    unsigned int exitc;   // blocks that left a marching kernel (the last resets queue)
    double tres;          // ||b - A x||_2 after the solve (read back with the state)
};

template <typename T>
struct OpT {
    const T* __restrict__ c;    // centre diagonal (general operator only)
    const T* __restrict__ off;  // 6 off-diagonal arrays W,E,S,N,B,T, each n long
    int64_t n;
};

template <typename T>
struct VecsT {
    T* x;        // y in the preconditioned variable, x at the end
    const T* b;
    T* rh;       // r_hat_0
    T* r[2];     // r[0] the iterate's r, r[1] step (8)'s r until K5 has used it
    T* u[2];     // u[0] the iterate's u, u[1] step (5)'s u until K5 has used it
    T* v[2];
    T* s[2];
    T* w;
    T* t;
};

// Work decomposition of the marching kernels: (j,k) tiles of block.x by
// block.y cells, runs of `planes` i-planes; item = chunk * tiles + tile.
struct MarchCfg {
    dim3 block;
    int tiles_x = 1, tiles_y = 1;
    int planes = 1;
    int nitems = 1;
    size_t smem = 0;
    int cpt = 1;      // cells per thread along k (2: paired 16-byte copies, needs an even n2)
    int cpc = 1;      // plane runs per field component (items: tiles x cpc x components)
    // Slab decomposition (dare_slabs.cu): the first partial-sum slot of this
    // launch's items and the items of all launches that share the reduction
    // (0: this launch alone), and per operand input the planes below the
    // first and above the last plane of the slab, one per field component
    // (null: wrap / zero as usual).
    int item_base = 0;
    int nitems_total = 0;
    const void* halo[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
};

// ---- deterministic grid reduction -----------------------------------------
__device__ __forceinline__ int thread_linear() { return threadIdx.x + blockDim.x * threadIdx.y; }
__device__ __forceinline__ int block_linear() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ int blocks_total() { return gridDim.x * gridDim.y * gridDim.z; }

// Block reduction of Q values; thread 0 gets the sums. Fixed order.
template <int Q>
__device__ __forceinline__ void block_sum(double (&v)[Q], double* sh /* [32*Q] */) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
    const int tid = thread_linear();
    const int lane = tid & 31, wid = tid >> 5;
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) sh[q * 32 + wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x * blockDim.y + 31) >> 5;
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
// finish, after which tot[] holds the grid-wide sums (fixed summation order,
// so results are reproducible run to run).  `base` / `total`: the block's
// slot is base + its index, and the sums span `total` slots filled by this
// and earlier launches (0: this launch's blocks).
template <int Q>
__device__ bool grid_reduce(double (&v)[Q], double* __restrict__ partials, unsigned int* counter,
                            double (&tot)[Q], int base = 0, int total = 0) {
    __shared__ double sh[32 * kMaxQ];
    __shared__ bool is_last;
    const int span = total > 0 ? total : blocks_total();
    block_sum<Q>(v, sh);
    const int tid = thread_linear();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < Q; q++) partials[q * kMaxBlocks + base + block_linear()] = v[q];
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        is_last = (prev == (unsigned)span - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double a[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) a[q] = 0.;
    const int nt = blockDim.x * blockDim.y;
    for (int b = tid; b < span; b += nt) {
#pragma unroll
        for (int q = 0; q < Q; q++) a[q] += __ldcg(partials + q * kMaxBlocks + b);
    }
    block_sum<Q>(a, sh);
#pragma unroll
    for (int q = 0; q < Q; q++) tot[q] = a[q];
    if (tid == 0) *counter = 0u;
    return true;
}

// ---- host-side launch helpers (dare_bicgstab2.cu) -------------------------
// `max_items`: the partial-sum slots the launch may use (fewer when several
// launches share one reduction)
MarchCfg march_config(const dare_ctx* ctx, const GridDev& g, size_t elem, int max_items = kMaxBlocks);
int ensure_solver_ws(dare_system* s);

template <typename T>
VecsT<T> carve_vecs(T* base, int64_t n, T* x, const T* b);

template <typename T, bool UNIT>
int launch_init(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const OpT<T>& op, const VecsT<T>& vs,
                SolverState* st, double* partials);

template <typename T, bool UNIT>
int launch_iteration(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, int sblocks, const OpT<T>& op,
                     const VecsT<T>& vs, SolverState* st, double* partials, int par, cudaEvent_t* ev);

// `wait`: read the final state back before returning (otherwise, on the
// graph path, the caller enqueues more work and reads it back itself).
int finish_iterations(dare_ctx* ctx, const SolverState* st, SolverState* st_host);

template <typename T, bool UNIT>
int run_iterations(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, int sblocks, const OpT<T>& op,
                   const VecsT<T>& vs, SolverState* st, SolverState* st_host, double* partials, cudaGraphExec_t* ge,
                   int max_it, int check_every, int kid_base, bool wait = true);

int launch_true_residual(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const OpT<double>& op,
                         const double* x, const double* b, SolverState* st, double* partials, double* out);
int launch_fold(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const double* diag, double* invd, double* ahat,
                SolverState* st, double* partials);
// invd = 1 / diag and the folded off-diagonals rounded to FP32 (no FP64 copy)
int launch_fold32(dare_ctx* ctx, const GridDev& g, const MarchCfg& m, const double* diag, double* invd, float* ahat32,
                  SolverState* st, double* partials);
int launch_scale(dare_ctx* ctx, int64_t n, const double* invd, double* x);
// Apply step (10) when the solve stopped between it and the last kernel of
// its iteration (st_host: the final state read back)
template <typename T>
int finish_step10(dare_ctx* ctx, int64_t n, const SolverState& st_host, const SolverState* st, const VecsT<T>& vs);

}  // namespace dare_gpu

// Solver workspace, owned by a dare_system.
struct dare_solver_ws {
    int64_t n = 0;
    double* ahat = nullptr;      // 6 * n, Jacobi-folded off-diagonals
    double* invd = nullptr;      // n
    double* vec = nullptr;       // 11 * n work vectors
    double* partials = nullptr;  // kMaxQ * kMaxBlocks (+ scratch)
    dare_gpu::SolverState* st = nullptr;
    dare_gpu::SolverState* st_host = nullptr;  // pinned
    cudaGraphExec_t graph[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    dare_gpu::MarchCfg march;
    int stream_blocks = 0;
    // FP32 inner solver of the refinement driver (dare_mixed.cu)
    float* ahat32 = nullptr;     // 6 * n
    float* vec32 = nullptr;      // 12 * n (11 work vectors + the correction)
    double* r64 = nullptr;       // unused slot kept for layout stability
    dare_gpu::MarchCfg march32;
    // learned-preconditioner solver (dare_learned.cu)
    struct dare_learned_ws* learned = nullptr;
};

void dare_mixed_ws_free(dare_solver_ws* ws);
void dare_learned_ws_free(struct dare_learned_ws* lw);
int dare_bicgstab2_fp64(dare_system* s, const dare_solver_params* p, dare_solve_report* rep);
