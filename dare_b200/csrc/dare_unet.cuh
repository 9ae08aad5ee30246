// dare_unet.cuh -- types of the learned linear preconditioner shared by the
// network code (dare_unet.cu) and the learned solver (dare_learned.cu).
#pragma once

#include <cuda_bf16.h>

#include "dare_internal.cuh"

namespace dare_gpu {
namespace unet {

using bf16 = __nv_bfloat16;

constexpr int kLevels = 4;
constexpr int kLayers = 8;
constexpr int kTaps = 27;
constexpr int kThreads = 128;  // one CTA = 4 warps = the 128 TMEM lanes of an M=128 tile
constexpr int kTileM = 128;    // output rows (padded positions) per MMA tile
// warp-specialised forward convolution: 4 epilogue warps + producer + one MMA warp per M tile
constexpr int kEpiThreads = 128;
__host__ __device__ constexpr int fwd_threads(int mt) { return (5 + mt) * 32; }
constexpr int kMaxSlots = 8;   // staged-plane ring depth limit
// Rows of a staged plane segment, rounded to the 8-row core-matrix groups.
__host__ __device__ inline int round8(int rows) { return (rows + 7) / 8 * 8; }

// A level's activations live zero-padded, [(n0+2)][(n1+2)][(n2+2)] positions
// with ghosts kept at zero, so every 3^3 tap is a constant shift of the
// flattened padded position, and chunk-planar: the 8-channel chunk kc of
// position Q is 16 contiguous bytes at element act_off(total, Q, kc).  A plane
// segment of one chunk is then one contiguous run, staged by one bulk copy
// straight into the K-major operand layout of the MMAs (core matrices of
// 8 positions x 16 bytes).
__host__ __device__ inline int64_t act_off(int64_t total, int64_t Q, int kc) { return ((int64_t)kc * total + Q) * 8; }
// Rows past either end of a chunk plane that a staged segment may read (they
// feed only outputs that are not stored); the activation block keeps this
// many spare rows before its first array and after its last, and grids are
// limited to rows of W + 8 < kActSlackRows positions.
constexpr int64_t kActSlackRows = 8192;

struct Geom {
    int n0, n1, n2;   // internal cells
    int W;            // n2 + 2 (row length)
    int plane;        // (n1 + 2) * (n2 + 2)
    int64_t total;    // (n0 + 2) * plane
    int tiles;        // ceil(plane / 128): M tiles per plane
};

inline Geom make_geom(int n0, int n1, int n2) {
    Geom g;
    g.n0 = n0;
    g.n1 = n1;
    g.n2 = n2;
    g.W = n2 + 2;
    g.plane = (n1 + 2) * (n2 + 2);
    g.total = (int64_t)(n0 + 2) * g.plane;
    g.tiles = (g.plane + kTileM - 1) / kTileM;
    return g;
}

// The rows of one staged input plane: the 128 outputs plus a one-row and
// one-cell halo on either side in the flattened (j,k) plane.
__host__ __device__ inline int stage_rows(const Geom& g) { return kTileM + 2 * g.W + 2; }
// ... and for MT consecutive tiles
__host__ __device__ inline int fwd_rows(const Geom& g, int mt) { return mt * kTileM + 2 * g.W + 2; }
// Kernels with the three dk taps in the MMA's N dimension: D row m of a
// 128-row M tile is position P - 1 + m, and out(P + m - 1) = D[m-1][dk 0] +
// D[m][dk 1] + D[m+1][dk 2] for m = 1 .. 126, so M tiles overlap by two rows.
constexpr int kOutStride = 126;
// rows staged per input plane for MT such tiles: the (j) halo of W rows on
// either side, no (k) halo
__host__ __device__ inline int strip_rows(const Geom& g, int mt) { return (mt - 1) * kOutStride + kTileM + 2 * g.W; }
// Row pitch of a staged plane: rounded to 8 rows, then offset so that the
// 16-byte chunks of one row written by neighbouring threads fall into
// different shared-memory banks.
__host__ __device__ inline int row_pitch(int rows, int c) {
    return ((rows + 7) / 8) * 8 + (c == 16 ? 4 : (c == 32 ? 2 : 1));
}

struct LayerDef {
    int level, cin, cout;
};
constexpr LayerDef kDefs[kLayers] = {{0, 1, 16},  {1, 16, 32}, {2, 32, 64}, {3, 64, 64},
                                     {3, 64, 64}, {2, 64, 32}, {1, 32, 16}, {0, 16, 1}};
enum LayerId { ENC0 = 0, ENC1, ENC2, ENC3, DEC3, DEC2, DEC1, DEC0 };

enum { IN_BF16 = 0, IN_EMBED = 1 };                  // operand staging
enum { OUT_STORE = 0, OUT_ADDUP = 1, OUT_F32 = 2 };  // forward epilogue

struct LaunchCfg {
    bool ready = false;
    dim3 grid;
    size_t smem = 0;
    int ppc = 1;   // planes per CTA
    int tpg = 27;  // taps per CTA (weight gradient)
    int cols = 32; // TMEM columns
    int occ = 0;   // resident CTAs per SM
    int mt = 1;    // 128-position tiles per CTA step (forward)
    int slots = 4; // staged-plane ring depth (forward)
};

struct Layer {
    int level = 0, cin = 0, cout = 0;  // real channel counts
    int cink = 16, coutk = 16;          // kernel channel counts (>= 16)
    int nt = 16;                        // forward output-channel tile
    int ntb = 16;                       // data-gradient output-channel tile
    int64_t woff = 0, nparam = 0;
    bf16* wf = nullptr;                 // packed forward weights
    bf16* wb = nullptr;                 // packed data-gradient weights (flipped, transposed)
    LaunchCfg fwd, bwd, wgr;
};

}  // namespace unet
}  // namespace dare_gpu

struct dare_unet {
    dare_ctx* ctx = nullptr;
    int device = 0;            // for dare_unet_destroy, which does not touch ctx
    int n[3] = {0, 0, 0};      // the grid the convolutions run on
    int64_t ncell = 0;
    // Coarse-correction form: the network acts on the 2x restricted grid of
    // the system's grid `fine`, N(u) = u + P (U(R u)) with R the average of
    // the 8 children and P the nearest prolongation (no full-resolution
    // convolution); 0 for the full-resolution form N(u) = u + U(u).
    int coarse = 0;
    int fine[3] = {0, 0, 0};
    int64_t fine_ncell = 0;
    float* cbuf = nullptr;     // coarse form: R u and the network's output (2 ncell)
    float* fbuf = nullptr;     // coarse form: a fine (residual, error) pair before restriction (2 fine_ncell)
    dare_gpu::unet::Geom geo[dare_gpu::unet::kLevels];
    dare_gpu::unet::Layer layer[dare_gpu::unet::kLayers];
    int64_t nparam = 0;
    // parameters and optimiser state (FP32)
    float* w = nullptr;
    float* grad = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int64_t adam_t = 0;
    // activations (bf16, padded): forward
    dare_gpu::unet::bf16* S0 = nullptr;  // enc0 (+ prolonged dec1)
    dare_gpu::unet::bf16* P1 = nullptr;
    dare_gpu::unet::bf16* S1 = nullptr;
    dare_gpu::unet::bf16* P2 = nullptr;
    dare_gpu::unet::bf16* S2 = nullptr;
    dare_gpu::unet::bf16* P3 = nullptr;
    dare_gpu::unet::bf16* E3 = nullptr;
    // backward
    dare_gpu::unet::bf16* dS0 = nullptr;
    dare_gpu::unet::bf16* dD1 = nullptr;
    dare_gpu::unet::bf16* dS1 = nullptr;
    dare_gpu::unet::bf16* dD2 = nullptr;
    dare_gpu::unet::bf16* dS2 = nullptr;
    dare_gpu::unet::bf16* dD3 = nullptr;
    dare_gpu::unet::bf16* dE3 = nullptr;
    dare_gpu::unet::bf16* dP3 = nullptr;
    dare_gpu::unet::bf16* dP2 = nullptr;
    dare_gpu::unet::bf16* dP1 = nullptr;
    void* act_block = nullptr;            // one allocation for all of the above
    float* X0 = nullptr;                  // k_conv_in input with a 16-byte row pitch, when the caller's has none
    float* z = nullptr;                   // forward output during training
    float* g = nullptr;                   // dL/dz
    float* part = nullptr;                // weight-gradient partial sums
    size_t part_floats = 0;
    double* dscal = nullptr;              // [0] loss accumulator
    int* err = nullptr;                   // device error word (bounded waits)
    uint32_t wait_limit = 1u << 22;       // polls of the role-to-role waits (= tc::kWaitLimit; dare_unet_set_wait_limit)
    int debug_skip = 0;                   // one-shot test hook (dare_unet_debug_skip_plane)
    // training ring of (residual, error) pairs
    float* ring_r = nullptr;
    float* ring_e = nullptr;
    float* ring_en = nullptr;             // ||e||^2 per pair
    int ring_cap = 0, ring_size = 0, ring_next = 0;
    float* batch_r = nullptr;             // gathered minibatch
    float* batch_e = nullptr;
    int batch_cap = 0;
    double* sol = nullptr;                // scratch FP64 vectors for pair generation
    int64_t steps = 0, pairs_seen = 0;
    uint64_t rng = 0x9E3779B97F4A7C15ull;
};

namespace dare_gpu {
namespace unet {
// z = N(u) on the context's stream (no synchronisation); used by the solver.
// u and z live on the system's grid (the fine grid of a coarse-form network).
int apply(dare_unet* net, const float* u, float* z);
}  // namespace unet
}  // namespace dare_gpu
