// dare_internal.cuh -- shared types and helpers of the sm_100a implementation.
//
// Memory layout in HBM (one B200 holds a 512^3 FP64 system):
//   * fields: ghosted arrays, (nx+2g)(ny+2g)(nz+2g) doubles per time level,
//     last dimension fastest (Data/GridVector.inl:68-71 with N = 1);
//   * system: structure-of-arrays diagonals diag[slot][cell], slot order
//     CENTER, WEST, EAST, SOUTH, NORTH, BOTTOM, TOP, plus rhs and x, all over
//     internal cells only (the Tpetra row map, Trilinos.inl:467-504);
//   * solver work vectors over internal cells; scalars live on the device.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/dare_gpu.h"

namespace dare_gpu {

constexpr int kSlots = 7;

struct GridDev {             // passed by value to kernels
    int dim;
    int ng;
    int n[3];                 // internal resolution (1 when inactive)
    int gn[3];                // ghosted resolution
    int og[3];                // ghost offset per dimension (0 when inactive)
    int periodic[3];
    int64_t ncell;
    int64_t ncell_ghosted;
    double dx[3];
    double volume;
    double area[3];
    // Staggered representation (CartesianRepresentation.inl:33-76): one more
    // cell along a staggered, non-periodic direction, the cell width of the
    // base grid, and the domain starting half a cell earlier (origin = -dx/2;
    // 0 otherwise).
    int staggered[3];
    double origin[3];
    // Solver view of a system with several field components: the components
    // are stacked along i (n[0] = ncomp x the grid's n0, ncell likewise), each
    // component's planes wrapping among themselves on a periodic x.
    int ncomp = 1;
};

}  // namespace dare_gpu

namespace dare_gpu {
// kernel ids for the optional per-kernel event timing
enum KernelId : int {
    KID_ASSEMBLE = 0,
    KID_FOLD = 1,
    KID_INIT = 2,
    KID_STEP1 = 3,
    KID_STEP2 = 4,
    KID_STEP3 = 5,
    KID_STEP4 = 6,
    KID_STEP5 = 7,
    KID_FINAL = 8,
    KID_COUNT = 16
};
}  // namespace dare_gpu

struct dare_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int64_t launches = 0;
    // per-kernel CUDA-event timing (dare_ctx_set_profiling)
    int profiling = 0;
    cudaEvent_t ev[16] = {nullptr};
    double stat_ms[dare_gpu::KID_COUNT] = {0};
    int64_t stat_n[dare_gpu::KID_COUNT] = {0};
};

struct dare_grid {
    dare_ctx* ctx = nullptr;
    dare_gpu::GridDev dev{};
};

// Every handle records its device at creation: its destroy function uses
// that, never the context or grid it was made from, so handles may be
// destroyed in any order (a garbage collector's, for instance).
struct dare_field {
    dare_grid* grid = nullptr;
    int device = 0;
    int num_levels = 0;
    int ncomp = 1;                // components, stored component-major: level[l][c * ncell_ghosted + cell]
    double* level[8] = {nullptr};
};

struct dare_solver_ws;  // defined in dare_bicgstab2.cu
void dare_solver_ws_free(dare_solver_ws* ws);

struct dare_system {
    dare_grid* grid = nullptr;
    int device = 0;
    int ncomp = 1;               // field components (block-diagonal, one 7-point stencil each)
    dare_gpu::GridDev sdev{};    // the solver's view: components stacked along i
    int bc_type[6] = {0, 0, 0, 0, 0, 0};        // the faces' conditions of every component ...
    double bc_value[6] = {0, 0, 0, 0, 0, 0};
    // ... unless a component has its own (dare_system_set_bc_component):
    // per component, 6 faces each; empty until the first per-component call
    std::vector<int> bc_type_c;
    std::vector<double> bc_value_c;
    // A slab of a larger grid (dare_slabs.cu): x ends shared with a
    // neighbouring slab (bit 0 low, bit 1 high), whose faces are not folded.
    int xint = 0;
    double* diag = nullptr;   // [7][ncomp][ncell], component-major within a slot
    double* rhs = nullptr;    // [ncomp][ncell]
    double* x = nullptr;
    dare_solver_ws* ws = nullptr;
};

namespace dare_gpu {

// ---- error handling: never abort, record the message on the context ------
int set_error(dare_ctx* ctx, int code, const std::string& msg);
int check_cuda(dare_ctx* ctx, cudaError_t e, const char* what);
#define DARE_CUDA(ctx, call)                                              \
    do {                                                                   \
        cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) return ::dare_gpu::check_cuda(ctx, _e, #call); \
    } while (0)
#define DARE_LAUNCHED(ctx)                                                 \
    do {                                                                   \
        (ctx)->launches++;                                                 \
        cudaError_t _e = cudaGetLastError();                               \
        if (_e != cudaSuccess) return ::dare_gpu::check_cuda(ctx, _e, "kernel launch"); \
    } while (0)

// ---- index helpers -------------------------------------------------------
__host__ __device__ inline int64_t local_index(const GridDev& g, int i, int j, int k) {
    return ((int64_t)(i + g.og[0]) * g.gn[1] + (j + g.og[1])) * g.gn[2] + (k + g.og[2]);
}

// Neighbour ordinal in the internal numbering, wrapped on periodic
// dimensions; a removed (non-periodic boundary) or inactive neighbour maps to
// the cell itself so every access stays in bounds (its coefficient is 0).
__host__ __device__ inline void neighbour_ordinals(const GridDev& g, int i, int j, int k, int64_t c,
                                                    int64_t nb[7]) {
    const int64_t sx = (int64_t)g.n[1] * g.n[2], sy = g.n[2];
    nb[0] = c;
    nb[1] = i > 0 ? c - sx : (g.periodic[0] ? c + (int64_t)(g.n[0] - 1) * sx : c);
    nb[2] = i < g.n[0] - 1 ? c + sx : (g.periodic[0] ? c - (int64_t)(g.n[0] - 1) * sx : c);
    nb[3] = j > 0 ? c - sy : (g.periodic[1] ? c + (int64_t)(g.n[1] - 1) * sy : c);
    nb[4] = j < g.n[1] - 1 ? c + sy : (g.periodic[1] ? c - (int64_t)(g.n[1] - 1) * sy : c);
    nb[5] = k > 0 ? c - 1 : (g.periodic[2] ? c + (g.n[2] - 1) : c);
    nb[6] = k < g.n[2] - 1 ? c + 1 : (g.periodic[2] ? c - (g.n[2] - 1) : c);
}

inline int grid_blocks(const dare_ctx* ctx, int64_t work, int threads, int per_sm) {
    int64_t b = (work + threads - 1) / threads;
    int64_t cap = (int64_t)ctx->num_sms * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace dare_gpu
