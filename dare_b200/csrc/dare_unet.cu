// dare_unet.cu -- the learned linear preconditioner N(u) = u + U(u) of the
// Jacobi-folded system: network kernels, training, C ABI.
//
// Convolutions are implicit GEMMs on the tcgen05 tensor cores.  A level's
// activations are zero-padded and channels-last ([padded cell][C] bf16), so
// the 27 taps of a 3^3 kernel are constant shifts of the flattened padded
// position.  One CTA owns 128 consecutive padded positions of a (j,k) plane
// and marches along i: it keeps the input planes i-1, i, i+1 of its
// positions (plus the one-row halo of the plane) in a 4-slot shared-memory
// ring, so every input element is fetched from HBM about once per plane
// pass, and issues for each output plane 27 x (Cin/16) MMAs of
// M=128 x N x K=16 whose A operand is the staged plane at the tap's shift
// (only the descriptor's start address changes) and whose B operand is the
// packed weight tile of that tap.  The FP32 accumulator lives in TMEM,
// double-buffered: the epilogue of plane i-1 (tcgen05.ld, bf16 store, or
// the fused prolongation-add into the finer level, or the FP32 output
// z = u + acc) and the prefetch of plane i+2 overlap the MMAs of plane i.
//
// Weight gradients run the same staging with the reduction over positions:
// dW[t][co][ci] = sum_p dY[p][co] X[p + shift_t][ci] as an MMA with
// M = co (128 rows, rows >= Cout are ignored), N = Cin of one tap, K = 16
// positions, both operands MN-major straight from the staged planes; each
// CTA accumulates its planes in TMEM and writes one partial per CTA, summed
// in a fixed order afterwards (deterministic).  Data gradients are forward
// convolutions with flipped, transposed weights.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include <cudaTypedefs.h>

#include "dare_bicgstab2.cuh"
#include "dare_tc.cuh"
#include "dare_unet.cuh"

using namespace dare_gpu;
using namespace dare_gpu::unet;
using namespace dare_gpu::tc;

namespace dare_gpu {
namespace unet {

constexpr size_t kMaxSmem = 232448;  // 227 KB of opt-in shared memory per CTA

// ---------------------------------------------------------------------------
// operand staging: one plane segment of `rows` padded positions starting at
// flattened position Q0, as C/8 planes of 16-byte chunks with row pitch RP
// (chunk (kc, q) at byte (kc * RP + q) * 16).  Positions outside the array
// and rows q >= valid_rows read zero.
// IN_EMBED (C == 16) takes an FP32 vector over the internal cells as channel
// 0 (rounded to bf16) and zero elsewhere: the slot's other channels are
// zeroed once per kernel (stage_zero), the FP32 values land asynchronously
// in a raw 4-byte-per-row buffer, and stage_finish (run by the issuing
// thread after its cp.async wait) writes the bf16 channel-0 values.
// FP32 channel-0 rows q = first, first + stride, ... of a plane segment into
// the raw buffer.  The padded coordinates of a row are stepped from the
// previous one (one division per call, not per row).
__device__ __forceinline__ void embed_rows(float* raw, const float* __restrict__ in32, const Geom& g, int64_t Q0,
                                           int rows, int valid_rows, int first, int stride) {
    const int Jn = g.n1 + 2;
    int64_t Q = Q0 + first;
    int I = 0, J = 0, K = 0;
    bool have = false;
    for (int q = first; q < rows; q += stride, Q += stride) {
        if (!have && Q >= 0) {
            I = (int)(Q / g.plane);
            const int rem = (int)(Q - (int64_t)I * g.plane);
            J = rem / g.W;
            K = rem - J * g.W;
            have = true;
        }
        const bool ok = have && Q < g.total && q < valid_rows && I >= 1 && I <= g.n0 && J >= 1 && J <= g.n1 &&
                        K >= 1 && K <= g.n2;
        if (ok)
            cp4(raw + q, in32 + ((int64_t)(I - 1) * g.n1 + (J - 1)) * g.n2 + (K - 1));
        else
            raw[q] = 0.f;
        if (have) {
            K += stride;
            while (K >= g.W) {
                K -= g.W;
                if (++J == Jn) {
                    J = 0;
                    ++I;
                }
            }
        }
    }
}

template <int C, int MODE>
__device__ __forceinline__ void stage(uint8_t* slot, float* raw, const bf16* __restrict__ in,
                                      const float* __restrict__ in32, const Geom& g, int64_t Q0, int rows, int RP,
                                      int valid_rows) {
    if (MODE == IN_BF16) {
        constexpr int KC = C / 8;
        const int nent = rows * KC;
        for (int idx = threadIdx.x; idx < nent; idx += kThreads) {
            const int q = idx / KC, kc = idx - q * KC;
            const int64_t Q = Q0 + q;
            const bool v = Q >= 0 && Q < g.total && q < valid_rows;
            cp16(slot + ((size_t)kc * RP + q) * 16, in + act_off(g.total, v ? Q : 0, kc), v);
        }
    } else {
        embed_rows(raw, in32, g, Q0, rows, valid_rows, threadIdx.x, kThreads);
    }
}

template <int MODE>
__device__ __forceinline__ void stage_finish(uint8_t* slot, const float* raw, int rows) {
    if (MODE == IN_EMBED) {
        for (int q = threadIdx.x; q < rows; q += kThreads)
            *reinterpret_cast<bf16*>(slot + (size_t)q * 16) = __float2bfloat16_rn(raw[q]);
    }
}

__device__ __forceinline__ void stage_zero(uint8_t* p, uint32_t bytes, int nthreads = kThreads) {
    for (uint32_t o = threadIdx.x * 16; o < bytes; o += nthreads * 16)
        *reinterpret_cast<uint4*>(p + o) = make_uint4(0u, 0u, 0u, 0u);
}

// The same staging done by one warp (lane-strided), for the producer warp of
// the warp-specialised forward kernel.
template <int C, int MODE>
__device__ __forceinline__ void stage_lanes(uint8_t* slot, float* raw, const bf16* __restrict__ in,
                                            const float* __restrict__ in32, const Geom& g, int64_t Q0, int rows,
                                            int RP, int lane) {
    if (MODE == IN_BF16) {
        constexpr int KC = C / 8;
        const int nent = rows * KC;
        for (int idx = lane; idx < nent; idx += 32) {
            const int q = idx / KC, kc = idx - q * KC;
            const int64_t Q = Q0 + q;
            const bool v = Q >= 0 && Q < g.total;
            cp16(slot + ((size_t)kc * RP + q) * 16, in + act_off(g.total, v ? Q : 0, kc), v);
        }
    } else {
        embed_rows(raw, in32, g, Q0, rows, rows, lane, 32);
    }
}

template <int MODE>
__device__ __forceinline__ void stage_finish_lanes(uint8_t* slot, const float* raw, int rows, int lane) {
    if (MODE == IN_EMBED) {
        for (int q = lane; q < rows; q += 32)
            *reinterpret_cast<bf16*>(slot + (size_t)q * 16) = __float2bfloat16_rn(raw[q]);
    }
}

// raw FP32 staging bytes of one slot (IN_EMBED), 16-byte aligned
__host__ __device__ inline uint32_t raw_bytes(int rows) { return (uint32_t)(((rows + 3) / 4) * 16); }

// ---------------------------------------------------------------------------
// forward convolution
struct FwdArgs {
    Geom g;          // level of input and output
    Geom fg;         // finer level (OUT_ADDUP)
    const bf16* in;  // [g.total][CIN]
    const bf16* w;   // packed [nz][9 (di,dj)][CIN/8][3 dk][NT][8]
    int cout;        // channel count (stride) of out / fine
    bf16* out;       // OUT_STORE: [g.total][cout]
    bf16* fine;      // OUT_ADDUP: [fg.total][cout]
    int ppc;
    int slots;       // ring depth (shared-memory slots of staged planes)
    int* err;
    uint32_t wait_limit;   // polls of the role-to-role waits (role_wait)
    int skip_plane;        // test hook: CTA 0 leaves its first plane unstaged
};

// Bounded mbarrier wait between the roles of a CTA (producer, MMA issuer,
// epilogue) that also gives up when another role has aborted.  `limit` polls
// (the network's run-time wait limit, kWaitLimit by default).  The waits of a
// role for its own asynchronous work (its MMAs, its copies in flight) keep
// the default limit, so an aborting CTA still releases TMEM and shared memory
// only after that work has landed.
__device__ __forceinline__ bool role_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                          int code, uint32_t limit) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < limit; it++) {
        if (mbar_try_wait(addr, parity)) return true;
        if ((it & 63) == 63 && *abort_flag) return false;
    }
    *abort_flag = 1;
    if (err) atomicCAS(err, 0, code);
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// One arrival per warp, by lane 0 once the whole warp got here: the barriers
// that collect a role's warps count warps, not threads (an arrival by every
// thread serialises on the barrier's word, ~1 us per plane for 512 of them).
__device__ __forceinline__ void warp_arrive(uint64_t* bar) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(bar);
}

template <int N>
__device__ __forceinline__ void cp_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// true in every epilogue thread if it is true in any (named barrier 1, the
// 128 epilogue threads)
__device__ __forceinline__ bool epi_any(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

// Offset (in cells) of child ch = 4 a + 2 b + c of a coarse cell from its
// first child on the finer level f: (+a planes, +b rows, +c cells).
__device__ __forceinline__ int64_t child_off(const Geom& f, int64_t fplane, int ch) {
    return (ch >> 2) * fplane + ((ch >> 1) & 1) * f.W + (ch & 1);
}

// Warp-specialised forward convolution with the three dk taps of a (di, dj)
// in the N dimension of one MMA: D[m][dk NT + co] = sum_{di,dj,ci}
// X[m + (di, dj)][ci] W[(di,dj,dk)][co][ci] over CIN/16 K steps per (di, dj),
// i.e. 9 x CIN/16 MMAs of N = 3 NT per 128-row tile (an MMA of M = 128, K = 16
// costs about the same for every N up to ~64, so this is ~3x fewer tensor
// cycles than one MMA per tap), and out(m) = D[m-1][dk 0] + D[m][dk 1] +
// D[m+1][dk 2] for m = 1 .. 126 (warp shuffles; the rows at a warp's edge
// come through shared memory).
// Roles: warps 0-3 drain the accumulators (each its 32-lane TMEM quarter),
// one lane of warp 4 stages input planes with TMA, one lane of each of warps
// 5 .. 5+MT-1 issues the MMAs of one M tile.  A CTA owns MT overlapping M
// tiles (126 outputs each) of a (j,k) plane and marches along i through
// planes I0..I1; input planes live in a ring of `slots` shared-memory slots,
// each CIN/8 chunk planes of RP rows x 16 bytes filled by TMA boxes of
// 8 channels x BR positions (rows outside the array read zero).
// Barriers:
//   full[s]   producer -> MMA   expect_tx + the boxes' bytes of slot s
//   empty[s]  MMA -> producer   the last MMAs reading slot s have completed (MT commits)
//   accf[b]   MMA -> epilogue   accumulator b holds a finished plane (MT commits)
//   acce[b]   epilogue -> MMA   accumulator b has been read (128 arrivals)
// Every wait is bounded; a role that times out raises a shared abort flag
// the others poll, and the MMA lane waits for its own MMAs before TMEM is
// released.  OUT_ADDUP (nearest-neighbour prolongation added into the eight
// children on the finer level) loads the children of plane I+1 while plane
// I+1's MMAs run.
template <int CIN, int NT, int MT, int OUTM>
__global__ void __launch_bounds__(fwd_threads(MT)) k_conv_fwd(FwdArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int KC = CIN / 8;
    constexpr int N3 = 3 * NT;
    constexpr uint32_t WB = kTaps * CIN * NT * 2;
    constexpr uint32_t AST = N3 <= 64 ? 64 : 128;  // TMEM columns of one tile's accumulator
    constexpr uint32_t ACOLS = MT * AST;           // ... of one buffer (two buffers)
    constexpr uint32_t COLS = 2 * ACOLS <= 128 ? 128 : (2 * ACOLS <= 256 ? 256 : 512);
    static_assert(2 * ACOLS <= 512, "accumulators exceed TMEM");
    static_assert(OUTM == OUT_STORE || OUTM == OUT_ADDUP, "forward epilogue");
    constexpr int XN = MT * 4 * 2 * NT;  // exchange floats per buffer
    const Geom g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int S = a.slots;
    const int RP = round8(strip_rows(g, MT));  // staged rows per chunk plane
    const uint32_t SB = (uint32_t)KC * RP * 16;
    uint8_t* wsm = smem;
    uint8_t* slots = smem + WB;
    float* exch = reinterpret_cast<float*>(slots + S * SB);  // [2][MT][4 warps][2][NT]
    uint64_t* bars = reinterpret_cast<uint64_t*>(exch + 2 * XN);
    uint64_t* full = bars;  // [kMaxSlots]
    uint64_t* empty = bars + kMaxSlots;
    uint64_t* accf = bars + 2 * kMaxSlots;
    uint64_t* acce = accf + 2;
    uint64_t* drain = acce + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

    const int P0 = blockIdx.x * (MT * kOutStride);
    const int I0 = 1 + blockIdx.y * a.ppc;
    if (I0 > g.n0) return;
    const int I1 = min(g.n0, I0 + a.ppc - 1);
    const int co0 = blockIdx.z * NT;

    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], MT);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&accf[b], MT);
            mbar_init(&acce[b], kEpiThreads / 32);
        }
        mbar_init(drain, MT);
        *abort_flag = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tslot, COLS);
    {
        const uint8_t* src = reinterpret_cast<const uint8_t*>(a.w) + (size_t)blockIdx.z * WB;
        for (uint32_t o = tid * 16; o < WB; o += fwd_threads(MT) * 16) cp16(wsm + o, src + o, true);
        cp_commit();
        cp_wait_all();
    }
    fence_proxy_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    // slot row 0 is position P0 - 1 - W; D row m of tile mt (position
    // P0 - 1 + 126 mt + m) reads slot rows 126 mt + m + dj W
    const int pbase = P0 - 1 - g.W;

    if (warp == 4) {
        // ---- producer: planes I0-1 .. I1+1 into the ring, one bulk copy per
        // chunk plane segment ----
        if (lane == 0) {
            const uint32_t bytes = (uint32_t)KC * RP * 16;
            uint32_t eph = 0xFFu;  // parity of the next wait on empty[s] (fresh slots pass)
            uint32_t armed = 0, apar = 0;  // slots armed so far; parity of each slot's next full phase
            // test hook (dare_unet_debug_skip_plane): the first CTA leaves its
            // first plane unstaged -- no arrive, no copies -- so the MMA
            // issuer's bounded wait for it runs out and the CTA aborts
            const bool skip = a.skip_plane && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0;
            for (int p = I0 - 1; p <= I1 + 1; p++) {
                const int sl = p % S;
                if (!role_wait(&empty[sl], (eph >> sl) & 1u, abort_flag, a.err, 5, a.wait_limit)) break;
                eph ^= 1u << sl;
                if (skip && p == I0 - 1) continue;
                mbar_arrive_expect_tx(&full[sl], bytes);
                armed |= 1u << sl;
                apar ^= 1u << sl;
                const int64_t y0 = (int64_t)p * g.plane + pbase;
                for (int kc = 0; kc < KC; kc++)
                    bulk_load(slots + sl * SB + (size_t)kc * RP * 16, a.in + act_off(g.total, y0, kc),
                              (uint32_t)RP * 16, &full[sl]);
            }
            // the copies in flight land before the CTA releases its shared
            // memory: wait for the last phase armed on every slot (already
            // complete unless the CTA is aborting)
            for (int sl = 0; sl < S; sl++)
                if ((armed >> sl) & 1u) mbar_wait(&full[sl], ((apar >> sl) & 1u) ^ 1u, nullptr, 0);
        }
        __syncwarp();
    } else if (warp >= 5) {
        // ---- MMA issue: lane 0 of warp 5 + mt, M tile mt ----
        const int mt = warp - 5;
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(kTileM, N3, 0, 0);
            const uint32_t sl0 = smem_u32(slots), wa = smem_u32(wsm);
            const uint64_t adesc = smem_desc(0, RP * 16, 128), bdesc = smem_desc(0, N3 * 16, 128);
            const uint32_t w16 = (uint32_t)g.W * 16, rp32 = (uint32_t)RP * 32;
            uint32_t fph = 0, aph = 3u;
            bool ok = true;
            for (int I = I0; I <= I1 && ok; I++) {
                const int buf = (I - I0) & 1;
                for (int p = (I == I0 ? I0 - 1 : I + 1); p <= I + 1 && ok; p++) {
                    const int sp = p % S;
                    ok = role_wait(&full[sp], (fph >> sp) & 1u, abort_flag, a.err, 6, a.wait_limit);
                    fph ^= 1u << sp;
                }
                if (ok) ok = role_wait(&acce[buf], (aph >> buf) & 1u, abort_flag, a.err, 7, a.wait_limit);
                aph ^= 1u << buf;
                if (!ok) break;
                fence_after_sync();
                // descriptors = constant high bits | (start address >> 4)
                const uint32_t sb[3] = {sl0 + (uint32_t)((I - 1) % S) * SB, sl0 + (uint32_t)(I % S) * SB,
                                        sl0 + (uint32_t)((I + 1) % S) * SB};
#pragma unroll
                for (int g9 = 0; g9 < 9; g9++) {
                    const int di = g9 / 3, dj = g9 % 3;
                    const uint32_t ab = sb[di] + dj * w16 + (uint32_t)(mt * kOutStride) * 16;
#pragma unroll
                    for (int s = 0; s < CIN / 16; s++)
                        mma_bf16(tmem + buf * ACOLS + mt * AST, adesc | (((ab + s * rp32) >> 4) & 0x3FFFu),
                                 bdesc | (((wa + (uint32_t)((g9 * KC + 2 * s) * N3 * 16)) >> 4) & 0x3FFFu), idesc,
                                 (g9 | s) ? 1u : 0u);
                }
                mma_commit(smem_u32(&accf[buf]));
                mma_commit(smem_u32(&empty[(I - 1) % S]));  // plane I-1 is not read again
            }
            // every MMA of this CTA (all issuers) has completed before TMEM is released
            mma_commit(smem_u32(drain));
            mbar_wait(drain, 0, a.err, 8);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warps 0-3; thread tid drains D row tid of every tile ----
        int pos[MT];  // in-plane output position of this thread's row, -1 if none
        int64_t fofs[MT];
        const Geom& f = a.fg;
        const int64_t fplane = (int64_t)(f.n1 + 2) * f.W;
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
            const int pp = P0 + mt * kOutStride + tid - 1;
            const int J = pp / g.W, K = pp - J * g.W;
            const bool ok = tid >= 1 && tid <= kOutStride && pp < g.plane && J >= 1 && J <= g.n1 && K >= 1 && K <= g.n2;
            pos[mt] = ok ? pp : -1;
            fofs[mt] = (int64_t)(2 * J - 1) * f.W + (2 * K - 1);  // first child, without the plane term (ADDUP)
        }
        // ADDUP: the children of the next plane are loaded ahead when their
        // registers fit (MT x NT <= 32), else just before their update
        constexpr bool kPre = OUTM == OUT_ADDUP && MT * NT <= 32;
        uint4 pre[kPre ? MT : 1][NT / 8][8];
        auto fetch = [&](int I, int mt, uint4(&o)[NT / 8][8]) {
            const int64_t Q = (int64_t)(2 * I - 1) * fplane + fofs[mt];
#pragma unroll
            for (int c8 = 0; c8 < NT / 8; c8++)
#pragma unroll
                for (int ch = 0; ch < 8; ch++)
                    o[c8][ch] = *reinterpret_cast<const uint4*>(
                        a.fine + act_off(f.total, Q + child_off(f, fplane, ch), co0 / 8 + c8));
        };
        if constexpr (kPre) {
#pragma unroll
            for (int mt = 0; mt < MT; mt++)
                if (pos[mt] >= 0) fetch(I0, mt, pre[mt]);
        }
        uint32_t fph = 0;
        for (int I = I0; I <= I1; I++) {
            const int buf = (I - I0) & 1;
            const bool ok = role_wait(&accf[buf], (fph >> buf) & 1u, abort_flag, a.err, 9, a.wait_limit);
            if (epi_any(!ok)) break;  // the four warps leave together
            fph ^= 1u << buf;
            fence_after_sync();
            float acc[MT][NT];
            float* ex = exch + buf * XN;
#pragma unroll
            for (int mt = 0; mt < MT; mt++)
#pragma unroll
                for (int c = 0; c < NT; c += 16) {
                    uint32_t r0[16], r1[16], r2[16];
                    const uint32_t t0 = tmem + ((uint32_t)(warp * 32) << 16) + buf * ACOLS + mt * AST + c;
                    tmem_ld16(t0, r0);
                    tmem_ld16(t0 + NT, r1);
                    tmem_ld16(t0 + 2 * NT, r2);
                    tmem_wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        reg_fence(r0[i]);
                        reg_fence(r1[i]);
                        reg_fence(r2[i]);
                        const float v0 = __shfl_up_sync(0xFFFFFFFFu, __uint_as_float(r0[i]), 1);
                        const float v2 = __shfl_down_sync(0xFFFFFFFFu, __uint_as_float(r2[i]), 1);
                        acc[mt][c + i] = (lane == 0 ? 0.f : v0) + __uint_as_float(r1[i]) + (lane == 31 ? 0.f : v2);
                    }
                    // the rows at the warp's edges feed the neighbouring warps
                    if (lane == 31) {
                        float4* e = reinterpret_cast<float4*>(ex + ((mt * 4 + warp) * 2 + 0) * NT + c);
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            e[i] = make_float4(__uint_as_float(r0[4 * i]), __uint_as_float(r0[4 * i + 1]),
                                               __uint_as_float(r0[4 * i + 2]), __uint_as_float(r0[4 * i + 3]));
                    } else if (lane == 0) {
                        float4* e = reinterpret_cast<float4*>(ex + ((mt * 4 + warp) * 2 + 1) * NT + c);
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            e[i] = make_float4(__uint_as_float(r2[4 * i]), __uint_as_float(r2[4 * i + 1]),
                                               __uint_as_float(r2[4 * i + 2]), __uint_as_float(r2[4 * i + 3]));
                    }
                }
            fence_before_sync();
            warp_arrive(&acce[buf]);
            epi_sync();  // the edge rows are in `ex` (double-buffered: the next plane writes the other half)
            if ((lane == 0 && warp > 0) || (lane == 31 && warp < 3)) {
                const int src = lane == 0 ? ((warp - 1) * 2 + 0) : ((warp + 1) * 2 + 1);
#pragma unroll
                for (int mt = 0; mt < MT; mt++)
#pragma unroll
                    for (int c = 0; c < NT; c++) acc[mt][c] += ex[(mt * 4 * 2 + src) * NT + c];
            }
#pragma unroll
            for (int mt = 0; mt < MT; mt++) {
                if (pos[mt] < 0) continue;
                if constexpr (OUTM == OUT_STORE) {
                    const int64_t Q = (int64_t)I * g.plane + pos[mt];
#pragma unroll
                    for (int c = 0; c < NT; c += 8)
                        *reinterpret_cast<uint4*>(a.out + act_off(g.total, Q, (co0 + c) / 8)) =
                            make_uint4(pack_bf16(acc[mt][c + 0], acc[mt][c + 1]), pack_bf16(acc[mt][c + 2], acc[mt][c + 3]),
                                       pack_bf16(acc[mt][c + 4], acc[mt][c + 5]), pack_bf16(acc[mt][c + 6], acc[mt][c + 7]));
                } else {
                    if constexpr (!kPre) fetch(I, mt, pre[0]);
                    const int64_t Q = (int64_t)(2 * I - 1) * fplane + fofs[mt];
#pragma unroll
                    for (int c8 = 0; c8 < NT / 8; c8++)
#pragma unroll
                        for (int ch = 0; ch < 8; ch++) {
                            const uint4 o = pre[kPre ? mt : 0][c8][ch];
                            const float* v = &acc[mt][c8 * 8];
                            *reinterpret_cast<uint4*>(a.fine + act_off(f.total, Q + child_off(f, fplane, ch),
                                                                       co0 / 8 + c8)) =
                                make_uint4(pack_bf16(bf16_lo(o.x) + v[0], bf16_hi(o.x) + v[1]),
                                           pack_bf16(bf16_lo(o.y) + v[2], bf16_hi(o.y) + v[3]),
                                           pack_bf16(bf16_lo(o.z) + v[4], bf16_hi(o.z) + v[5]),
                                           pack_bf16(bf16_lo(o.w) + v[6], bf16_hi(o.w) + v[7]));
                        }
                }
            }
            if constexpr (kPre) {
                if (I < I1) {
#pragma unroll
                    for (int mt = 0; mt < MT; mt++)
                        if (pos[mt] >= 0) fetch(I + 1, mt, pre[mt]);
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, COLS);
    }
}

// ---------------------------------------------------------------------------
// One-channel layers.  A tcgen05 MMA of M = 128, K = 16 costs about the same
// for any N up to ~64 (measured: ~42 cycles per MMA when the SM's pipe is
// saturated, ~55 from a single issuing thread), so the 3^3 convolutions with
// a single input or output channel are re-cast so that each MMA carries
// several taps:
//   k_conv_in  (1 -> 16, FP32 input): 2-D tiles of 16 rows j x 8 cells k and
//              "window" rows holding the six taps (dj, dj + 1) x (dk 0..2) of
//              one output cell in a K-chunk of 8; the chunk two rows j further
//              holds dj = 2, and N = 3 di x 16 output channels: one MMA per
//              tile and input plane, whose accumulator holds the partial sums
//              of the three output planes that input plane feeds.
//   k_conv_out (16 -> 1, FP32 output): N = (di, dk) (9 of 16 columns),
//              3 MMAs (one per dj) per input plane and 126 outputs; the dk
//              terms meet across neighbouring rows in the epilogue.

// Both kernels read each input plane's accumulator once, into running sums
// of the output planes it still feeds.  A test of an already completed
// mbarrier phase was measured at 250-500 cycles, and every role pays two or
// three per round of its loop, so the loops are latency-bound: k_conv_in
// takes its planes two per round, while k_conv_out (whose staged planes are
// ~25 KB at 256^2) gains more from CTAs per SM than from groups (measured at
// 256^3: groups of two with a 2-group ring 242 us, single planes with 3 CTAs
// per SM 183 us).

// k_conv_out: planes per group, and accumulator groups
constexpr int kOutB = 1;
constexpr int kOutG = 4;

// k_conv_in: an M tile is 16 rows j x 8 cells k of a plane (row m = 8 g + t:
// j = j0 + g, k = 8 kb + t), a CTA covers MT tiles stacked in j and marches a
// run of planes, kInB planes at a time: every role pays its mbarrier
// round trips (measured at 250-500 cycles for the test of an already
// completed phase, so each role's loop is bound by their latency) once per
// group.  Per group a TMA box of the FP32 input (cells k = 8 kb - 4 ..
// 8 kb + 11, rows j0 - 1 .. j0 + 16 MT + 1, kInB planes; cells outside the
// grid read zero, which are the ghost values) lands in a ring of kInRaw
// slots; builder warps turn it into 16 MT + 2 window rows per k and plane
// (BF16, a ring of kInWin slots), and one MMA per tile and plane multiplies a
// window plane with the packed weights.  The epilogue reads each plane's
// accumulator once, into running sums of the two output planes it still
// feeds; 8 epilogue warps (two per TMEM lane quarter) take 8 output channels
// each.
constexpr int kInB = 2;            // planes per group
constexpr int kInRaw = 8;          // staged FP32 boxes (groups)
constexpr int kInWin = 3;          // window groups
constexpr int kInAcc = 2;          // accumulator groups
constexpr int kInEpi = 256;        // epilogue threads (8 warps)
constexpr int kInBuilders = 128;   // window builder threads (4 warps)
constexpr int kInBoxK = 16;        // FP32 cells per box row
constexpr uint32_t kInWB = 2 * 48 * 16;  // packed weights [2 chunks][3 di x 16 co][8] bf16, bytes

struct InArgs {
    Geom g;
    const bf16* w;      // [2 chunks][3 di x 16 co][8]: chunk c, element e < 6: dj = 2 c + e / 3, dk = e % 3
    bf16* out;          // chunk-planar [2][g.total][8]
    bf16* pool;         // if set: pool_scale x (sum of the 2x2x2 children of `out`), chunk-planar on level cg
    Geom cg;
    float pool_scale;
    int ppc;            // even: a CTA's output planes start on an odd plane I and pair up
    int* err;
    uint32_t wait_limit;   // polls of the role-to-role waits (role_wait)
    CUtensorMap x;      // FP32 input [n0][n1][pitch >= n2], boxes kInBoxK x (16 MT + 3) x kInB
};

// 8 epilogue warps, 1 MMA warp, 4 window-builder warps, 1 producer warp
__host__ __device__ constexpr int in_threads() { return (8 + 1 + 4 + 1) * 32; }
__host__ __device__ constexpr int in_win_rows(int mt) { return 16 * mt + 2; }
__host__ __device__ constexpr uint32_t in_win_bytes(int mt) { return (uint32_t)in_win_rows(mt) * 8 * 16; }
// one plane of a box, and one box (kInB planes, 128-byte multiple)
__host__ __device__ constexpr uint32_t in_box_plane(int mt) { return (uint32_t)kInBoxK * (16 * mt + 3) * 4; }
__host__ __device__ constexpr uint32_t in_raw_stride(int mt) { return (kInB * in_box_plane(mt) + 127) / 128 * 128; }
__host__ __device__ constexpr size_t in_smem(int mt) {
    return kInRaw * (size_t)in_raw_stride(mt) + kInWin * (size_t)kInB * in_win_bytes(mt) + kInWB +
           (2 * kInRaw + 2 * kInWin + 2 * kInAcc + 1) * 8 + 16;
}

// enc0 forward and dec0 data gradient: 1 -> 16 channels.
template <int MT>
__global__ void __launch_bounds__(in_threads()) k_conv_in(const __grid_constant__ InArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr uint32_t AST = 64;                    // TMEM columns of one tile's accumulator (48 used)
    constexpr uint32_t ACOLS = MT * AST;            // one plane's accumulator (all tiles)
    constexpr uint32_t COLS = kInAcc * kInB * ACOLS;
    constexpr int WR = in_win_rows(MT);
    constexpr uint32_t WINB = in_win_bytes(MT), RAWS = in_raw_stride(MT), BOXP = in_box_plane(MT);
    const Geom g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t* raw = smem;                            // [kInRaw][RAWS]: FP32 [kInB][16 MT + 3][kInBoxK]
    uint8_t* win = raw + kInRaw * RAWS;             // [kInWin][kInB][WR][8 k][16 B]
    uint8_t* wsm = win + kInWin * kInB * WINB;
    uint64_t* bars = reinterpret_cast<uint64_t*>(wsm + kInWB);
    uint64_t* rawf = bars;                          // [kInRaw] box landed
    uint64_t* rawe = rawf + kInRaw;                 // [kInRaw] box read by the builders
    uint64_t* full = rawe + kInRaw;                 // [kInWin] window planes built
    uint64_t* empty = full + kInWin;                // [kInWin] window planes read by the MMAs
    uint64_t* accf = empty + kInWin;                // [kInAcc]
    uint64_t* acce = accf + kInAcc;                 // [kInAcc]
    uint64_t* drain = acce + kInAcc;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

    const int kbs = (g.n2 + 7) / 8;
    const int kb = blockIdx.x % kbs, jb = blockIdx.x / kbs;
    const int I0 = 1 + blockIdx.y * a.ppc;
    if (I0 > g.n0) return;
    const int I1 = min(g.n0, I0 + a.ppc - 1);
    const int np = I1 - I0 + 3;               // input planes I0 - 1 .. I1 + 1
    const int ng = (np + kInB - 1) / kInB;    // groups (the last one may run past I1 + 1)

    if (tid == 0) {
        for (int s = 0; s < kInRaw; s++) {
            mbar_init(&rawf[s], 1);
            mbar_init(&rawe[s], kInBuilders / 32);
        }
        for (int s = 0; s < kInWin; s++) {
            mbar_init(&full[s], kInBuilders / 32);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < kInAcc; b++) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], kInEpi / 32);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tslot, COLS);
    for (uint32_t o = tid * 16; o < kInWB; o += in_threads() * 16)
        cp16(wsm + o, reinterpret_cast<const uint8_t*>(a.w) + o, true);
    cp_commit();
    cp_wait_all();
    fence_proxy_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp == 13) {
        // ---- producer: one TMA box per group of planes ----
        if (lane == 0) {
            int q = 0;
            for (; q < ng; q++) {
                const int sl = q % kInRaw;
                if (!role_wait(&rawe[sl], ((q / kInRaw) & 1) ^ 1, abort_flag, a.err, 11, a.wait_limit)) break;
                mbar_arrive_expect_tx(&rawf[sl], kInB * BOXP);
                tma_load_3d(raw + sl * RAWS, &a.x, 8 * kb - 4, 16 * MT * jb - 1, I0 - 2 + kInB * q, &rawf[sl]);
            }
            // boxes still in flight land before the CTA leaves
            for (int r = max(0, q - kInRaw); r < q; r++) mbar_wait(&rawf[r % kInRaw], (r / kInRaw) & 1, nullptr, 0);
        }
        __syncwarp();
    } else if (warp >= 9) {
        // ---- window builders: row (jr, t) = x(jr, t-1..t+1), x(jr+1, t-1..t+1), 0, 0 ----
        const int bt = tid - 9 * 32;
        for (int q = 0; q < ng; q++) {
            const int sr = q % kInRaw, sw = q % kInWin;
            bool ok = role_wait(&rawf[sr], (q / kInRaw) & 1, abort_flag, a.err, 12, a.wait_limit);
            if (ok) ok = role_wait(&empty[sw], ((q / kInWin) & 1) ^ 1, abort_flag, a.err, 12, a.wait_limit);
            if (!__all_sync(0xffffffffu, ok)) break;  // the warp leaves together (__syncwarp below)
            const float* x = reinterpret_cast<const float*>(raw + sr * RAWS);
            uint8_t* wp = win + sw * kInB * WINB;
            for (int it = bt; it < kInB * WR * 8; it += kInBuilders) {
                // box cell e is k = 8 kb - 4 + e: output cell 8 kb + t reads e = t + 3 .. t + 5;
                // window rows of the group's planes follow each other as the box's planes do
                const float* r0 = x + (it >> 3) * kInBoxK + (it & 7) + 3 + (it / (WR * 8)) * kInBoxK;
                const float* r1 = r0 + kInBoxK;
                *reinterpret_cast<uint4*>(wp + it * 16) =
                    make_uint4(pack_bf16(r0[0], r0[1]), pack_bf16(r0[2], r1[0]), pack_bf16(r1[1], r1[2]), 0u);
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&full[sw]);
                mbar_arrive(&rawe[sr]);
            }
        }
    } else if (warp == 8) {
        // ---- MMA: one per tile and input plane, D_p[m][16 di + co] ----
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(kTileM, 48, 0, 0);
            const uint32_t w0 = smem_u32(win), wa = smem_u32(wsm);
            const uint64_t adesc = smem_desc(0, 2 * 128, 128);   // K chunk 1: two rows j further
            const uint64_t bdesc = smem_desc(0, 48 * 16, 128);
            bool ok = true;
            for (int q = 0; q < ng && ok; q++) {
                const int sw = q % kInWin, ab = q & (kInAcc - 1);
                ok = role_wait(&full[sw], (q / kInWin) & 1, abort_flag, a.err, 13, a.wait_limit);
                if (ok) ok = role_wait(&acce[ab], ((q / kInAcc) & 1) ^ 1, abort_flag, a.err, 14, a.wait_limit);
                if (!ok) break;
                fence_after_sync();
#pragma unroll
                for (int b = 0; b < kInB; b++)
#pragma unroll
                    for (int mt = 0; mt < MT; mt++) {
                        const uint32_t a0 = w0 + (uint32_t)(sw * kInB + b) * WINB + (uint32_t)mt * 16 * 128;
                        mma_bf16(tmem + (ab * kInB + b) * ACOLS + mt * AST, adesc | ((a0 >> 4) & 0x3FFFu),
                                 bdesc | ((wa >> 4) & 0x3FFFu), idesc, 0u);
                    }
                mma_commit(smem_u32(&accf[ab]));
                mma_commit(smem_u32(&empty[sw]));
            }
            mma_commit(smem_u32(drain));
            mbar_wait(drain, 0, a.err, 16);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 and output
        // channels 8 (w / 4) .. + 7 of those rows ----
        const int qd = warp & 3, h = warp >> 2, m = 32 * qd + lane;
        int64_t pos[MT];  // in-plane output position of this thread's row, -1 if none
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
            const int jo = 16 * MT * jb + 16 * mt + (m >> 3), ko = 8 * kb + (m & 7);
            pos[mt] = jo < g.n1 && ko < g.n2 ? (int64_t)(jo + 1) * g.W + ko + 1 : -1;
        }
        // input plane p = I0 - 1 + k feeds outputs p + 1 (di 0), p (di 1) and
        // p - 1 (di 2); before it, cur holds the partial sum of output p - 1
        // (planes p - 2 and p - 1) and nxt that of output p (plane p - 1)
        float cur[MT][8] = {}, nxt[MT][8] = {};
        float pooled[MT][8];  // 2x2 sum of the first (odd) plane of a pair, on the lanes with j, k even
        for (int q = 0; q < ng; q++) {
            const int ab = q & (kInAcc - 1);
            const bool okw = role_wait(&accf[ab], (q / kInAcc) & 1, abort_flag, a.err, 17, a.wait_limit);
            if (!__all_sync(0xffffffffu, okw)) break;  // tcgen05.ld below is warp-collective
            fence_after_sync();
            uint32_t r[kInB][MT][3][8];
#pragma unroll
            for (int b = 0; b < kInB; b++)
#pragma unroll
                for (int mt = 0; mt < MT; mt++)
#pragma unroll
                    for (int di = 0; di < 3; di++)
                        tmem_ld8(tmem + ((uint32_t)(32 * qd) << 16) + (ab * kInB + b) * ACOLS + mt * AST + 16 * di +
                                     8 * h,
                                 r[b][mt][di]);
            tmem_wait_ld();
            fence_before_sync();
            warp_arrive(&acce[ab]);
#pragma unroll
            for (int b = 0; b < kInB; b++) {
                const int k = kInB * q + b;
                const int I = I0 - 2 + k;  // output completed by this plane
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
                    float o[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        reg_fence(r[b][mt][0][c]);
                        reg_fence(r[b][mt][1][c]);
                        reg_fence(r[b][mt][2][c]);
                        o[c] = cur[mt][c] + __uint_as_float(r[b][mt][2][c]);
                        cur[mt][c] = nxt[mt][c] + __uint_as_float(r[b][mt][1][c]);
                        nxt[mt][c] = __uint_as_float(r[b][mt][0][c]);
                    }
                    if (k >= 2 && k < np) {
                        const uint4 ov = make_uint4(pack_bf16(o[0], o[1]), pack_bf16(o[2], o[3]),
                                                    pack_bf16(o[4], o[5]), pack_bf16(o[6], o[7]));
                        if (pos[mt] >= 0) {
                            const int64_t Q = (int64_t)I * g.plane + pos[mt];
                            *reinterpret_cast<uint4*>(a.out + act_off(g.total, Q, h)) = ov;
                        }
                        if (a.pool) {
                            // the children in the order of k_restrict: planes I, I + 1; in
                            // each, (j, k), (j, k+1), (j+1, k), (j+1, k+1) -- lanes +0, +1, +8, +9.
                            // I0 is odd and a group holds an even number of planes, so
                            // output plane I is the second of its pair when b is odd.
                            static_assert(kInB % 2 == 0, "plane pairs must not straddle groups");
                            const bool second = (b & 1) != 0;
                            const float v[8] = {bf16_lo(ov.x), bf16_hi(ov.x), bf16_lo(ov.y), bf16_hi(ov.y),
                                                bf16_lo(ov.z), bf16_hi(ov.z), bf16_lo(ov.w), bf16_hi(ov.w)};
#pragma unroll
                            for (int c = 0; c < 8; c++) {
                                const float v1 = __shfl_down_sync(0xffffffffu, v[c], 1);
                                const float v8 = __shfl_down_sync(0xffffffffu, v[c], 8);
                                const float v9 = __shfl_down_sync(0xffffffffu, v[c], 9);
                                float acc = second ? pooled[mt][c] + v[c] : v[c];
                                acc += v1;
                                acc += v8;
                                acc += v9;
                                pooled[mt][c] = acc;
                            }
                            if (second && (lane & 9) == 0 && pos[mt] >= 0) {
                                const int jo = 16 * MT * jb + 16 * mt + (m >> 3), ko = 8 * kb + (m & 7);
                                const int64_t Qc =
                                    ((int64_t)((I - 2) / 2 + 1) * (a.cg.n1 + 2) + (jo / 2 + 1)) * a.cg.W + ko / 2 + 1;
                                const float sc = a.pool_scale;
                                *reinterpret_cast<uint4*>(a.pool + act_off(a.cg.total, Qc, h)) = make_uint4(
                                    pack_bf16(pooled[mt][0] * sc, pooled[mt][1] * sc),
                                    pack_bf16(pooled[mt][2] * sc, pooled[mt][3] * sc),
                                    pack_bf16(pooled[mt][4] * sc, pooled[mt][5] * sc),
                                    pack_bf16(pooled[mt][6] * sc, pooled[mt][7] * sc));
                            }
                        }
                    }
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, COLS);
    }
}

struct OutArgs {
    Geom g;
    const bf16* in;     // [g.total][16]
    const bf16* w;      // [9 (di,dj)][2 kc][16 n][8]: row n = dk < 3 holds W[(di,dj,dk)][0][8 kc ..]
    float* out32;       // internal cells
    const float* res32; // added to the output (may be null)
    int ppc, slots;
    int* err;
    uint32_t wait_limit;   // polls of the role-to-role waits (role_wait)
};

// 4 epilogue warps, producer, one MMA warp per M tile
__host__ __device__ constexpr int out_threads(int mt) { return (5 + mt) * 32; }

// dec0 forward: 16 -> 1 channel, z = res + conv.  Each staged INPUT plane p
// gets its own accumulator with the (di, dk) taps in N (N = 16, 9 used):
//     D_p[q][3 di + dk] = sum_dj sum_ci X_p[q + (dj-1) W][ci] W[(di,dj,dk)][ci]
// i.e. 3 MMAs per input plane (one per dj, whose shift is the A operand's
// start row).  Output plane I takes, for di = 0, 1, 2, the di columns of the
// accumulator of input plane I - 1 + di:
//     s_k(I)[m] = sum_di D_{I-1+di}[m][3 di + k]
//     out[m]    = s_0(I)[m-1] + s_1(I)[m] + s_2(I)[m+1]
// (m = 1 .. 126 of a 128-row tile).  The epilogue reads each accumulator once
// into running sums of s(p - 1), s(p) and s(p + 1); the three s_k of every row
// then meet their neighbours through shared memory.  Planes go kOutB to a
// group (one staged slot, one set of accumulators, one round of barriers).
template <int MT>
__global__ void __launch_bounds__(out_threads(MT)) k_conv_out(OutArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr uint32_t WB = 3 * 2 * 16 * 16;       // [3 dj][2 kc][16 n][8] bf16
    constexpr uint32_t ACOLS = MT * 16;            // one plane's accumulator (all tiles)
    constexpr uint32_t COLS = kOutG * kOutB * ACOLS <= 64 ? 64 : 128;
    const Geom g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int S = a.slots;                     // staged groups
    const int RP = round8(strip_rows(g, MT));  // staged rows per chunk plane
    const uint32_t SB = 2u * RP * 16;          // one staged plane
    uint8_t* wsm = smem;
    uint8_t* slots = smem + WB;                // [S][kOutB][2 kc][RP][16 B]
    float* dsm = reinterpret_cast<float*>(slots + S * kOutB * SB);  // [2][MT][128][3]
    uint64_t* bars = reinterpret_cast<uint64_t*>(dsm + 2 * MT * kTileM * 3);
    uint64_t* full = bars;
    uint64_t* empty = bars + kMaxSlots;
    uint64_t* accf = bars + 2 * kMaxSlots;       // [kOutG]
    uint64_t* acce = accf + kOutG;               // [kOutG]
    uint64_t* drain = acce + kOutG;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

    const int P0 = blockIdx.x * (MT * kOutStride);
    const int I0 = 1 + blockIdx.y * a.ppc;
    if (I0 > g.n0) return;
    const int I1 = min(g.n0, I0 + a.ppc - 1);
    const int np = I1 - I0 + 3;               // input planes I0 - 1 .. I1 + 1
    const int ng = (np + kOutB - 1) / kOutB;  // groups (the last one may run past I1 + 1)

    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], MT);
        }
        for (int b = 0; b < kOutG; b++) {
            mbar_init(&accf[b], MT);
            mbar_init(&acce[b], kEpiThreads / 32);
        }
        mbar_init(drain, MT);
        *abort_flag = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tslot, COLS);
    for (uint32_t o = tid * 16; o < WB; o += out_threads(MT) * 16)
        cp16(wsm + o, reinterpret_cast<const uint8_t*>(a.w) + o, true);
    cp_commit();
    cp_wait_all();
    fence_proxy_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    // segment row 0 is position P0 - 1 - W: D row m of tile mt (position
    // P0 - 1 + 126 mt + m) reads segment rows 126 mt + m + dj W
    const int pbase = P0 - 1 - g.W;

    if (warp == 4) {
        // ---- producer: one bulk copy per chunk plane segment; planes past
        // I1 + 1 in the last group are not copied (their slot keeps stale
        // rows whose accumulators are never read) ----
        if (lane == 0) {
            int q = 0;
            for (; q < ng; q++) {
                const int sl = q % S;
                if (!role_wait(&empty[sl], ((q / S) & 1) ^ 1, abort_flag, a.err, 21, a.wait_limit)) break;
                const int nb = min(kOutB, np - kOutB * q);
                mbar_arrive_expect_tx(&full[sl], (uint32_t)nb * 2u * RP * 16);
                for (int b = 0; b < nb; b++) {
                    const int64_t y0 = (int64_t)(I0 - 1 + kOutB * q + b) * g.plane + pbase;
                    for (int kc = 0; kc < 2; kc++)
                        bulk_load(slots + (size_t)(sl * kOutB + b) * SB + (size_t)kc * RP * 16,
                                  a.in + act_off(g.total, y0, kc), (uint32_t)RP * 16, &full[sl]);
                }
            }
            // the copies in flight land before the CTA releases its shared memory
            for (int r = max(0, q - S); r < q; r++) mbar_wait(&full[r % S], (r / S) & 1, nullptr, 0);
        }
        __syncwarp();
    } else if (warp >= 5) {
        // ---- MMA: 3 dj shifts per input plane, M tile mt = warp - 5 ----
        const int mt = warp - 5;
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(kTileM, 16, 0, 0);
            const uint32_t sl0 = smem_u32(slots), wa = smem_u32(wsm);
            const uint64_t adesc = smem_desc(0, RP * 16, 128), bdesc = smem_desc(0, 16 * 16, 128);
            const uint32_t w16 = (uint32_t)g.W * 16;
            bool ok = true;
            for (int q = 0; q < ng && ok; q++) {
                const int sl = q % S, ag = q & (kOutG - 1);
                ok = role_wait(&full[sl], (q / S) & 1, abort_flag, a.err, 22, a.wait_limit);
                if (ok) ok = role_wait(&acce[ag], ((q / kOutG) & 1) ^ 1, abort_flag, a.err, 23, a.wait_limit);
                if (!ok) break;
                fence_after_sync();
#pragma unroll
                for (int b = 0; b < kOutB; b++) {
                    const uint32_t ab = sl0 + (uint32_t)(sl * kOutB + b) * SB + (uint32_t)(mt * kOutStride) * 16;
#pragma unroll
                    for (int dj = 0; dj < 3; dj++)
                        mma_bf16(tmem + (ag * kOutB + b) * ACOLS + mt * 16, adesc | (((ab + dj * w16) >> 4) & 0x3FFFu),
                                 bdesc | (((wa + (uint32_t)(dj * 2 * 16 * 16)) >> 4) & 0x3FFFu), idesc,
                                 dj ? 1u : 0u);
                }
                mma_commit(smem_u32(&accf[ag]));
                mma_commit(smem_u32(&empty[sl]));
            }
            mma_commit(smem_u32(drain));
            mbar_wait(drain, 0, a.err, 24);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warps 0-3 ----
        int cof[MT];  // cell of this thread's output within a plane of internal cells, -1 if none
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
            const int pp = P0 + mt * kOutStride + tid;
            const int Jr = pp / g.W, Kc = pp - Jr * g.W;
            cof[mt] = tid < kOutStride && pp < g.plane && Jr >= 1 && Jr <= g.n1 && Kc >= 1 && Kc <= g.n2
                          ? (Jr - 1) * g.n2 + (Kc - 1)
                          : -1;
        }
        const int64_t cplane = (int64_t)g.n1 * g.n2;
        // the residual term of output plane I is loaded one plane ahead
        float res[MT];
        auto fetch = [&](int I) {
#pragma unroll
            for (int mt = 0; mt < MT; mt++)
                res[mt] = a.res32 && cof[mt] >= 0 ? a.res32[(int64_t)(I - 1) * cplane + cof[mt]] : 0.f;
        };
        fetch(I0);
        // input plane p = I0 - 1 + k: before it, cur holds the partial s of
        // output p - 1 (planes p - 2, p - 1) and nxt that of output p (plane p - 1)
        float cur[MT][3] = {}, nxt[MT][3] = {};
        for (int q = 0; q < ng; q++) {
            const int ag = q & (kOutG - 1);
            const bool okw = role_wait(&accf[ag], (q / kOutG) & 1, abort_flag, a.err, 25, a.wait_limit);
            if (epi_any(!okw)) break;  // the four warps leave together
            fence_after_sync();
            uint32_t r[kOutB][MT][16];
#pragma unroll
            for (int b = 0; b < kOutB; b++)
#pragma unroll
                for (int mt = 0; mt < MT; mt++)
                    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (ag * kOutB + b) * ACOLS + mt * 16, r[b][mt]);
            tmem_wait_ld();
            fence_before_sync();
            warp_arrive(&acce[ag]);
#pragma unroll
            for (int b = 0; b < kOutB; b++) {
                const int k = kOutB * q + b;
                const int I = I0 - 2 + k;  // output completed by this plane
                float* d = dsm + (k & 1) * MT * kTileM * 3;
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
#pragma unroll
                    for (int c = 0; c < 9; c++) reg_fence(r[b][mt][c]);
#pragma unroll
                    for (int kk = 0; kk < 3; kk++) {
                        d[(mt * kTileM + tid) * 3 + kk] = cur[mt][kk] + __uint_as_float(r[b][mt][6 + kk]);
                        cur[mt][kk] = nxt[mt][kk] + __uint_as_float(r[b][mt][3 + kk]);
                        nxt[mt][kk] = __uint_as_float(r[b][mt][kk]);
                    }
                }
                epi_sync();  // d[] complete (double-buffered: the next plane writes the other half)
                if (k >= 2 && k < np) {
#pragma unroll
                    for (int mt = 0; mt < MT; mt++) {
                        if (cof[mt] < 0) continue;
                        const float* dm = d + (mt * kTileM + tid) * 3;
                        a.out32[(int64_t)(I - 1) * cplane + cof[mt]] = res[mt] + (dm[0] + dm[3 + 1] + dm[6 + 2]);
                    }
                    if (I < I1) fetch(I + 1);
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, COLS);
    }
}

// ---------------------------------------------------------------------------
// weight gradient
struct WgrArgs {
    Geom g;
    const bf16* x;     // input activations (IN_BF16) ...
    const float* x32;  // ... or the FP32 vector (IN_EMBED)
    const bf16* dy;    // output gradient (IN_BF16) ...
    const float* dy32; // ... or the FP32 vector (IN_EMBED)
    float* part;       // [cta][tpg][COUT][CIN]
    int ppc, tpg;
    uint32_t cols;
    int* err;
    uint32_t wait_limit;   // polls of the role-to-role waits (role_wait)
};

template <int C>
__host__ __device__ constexpr int dy_pitch() {
    return kTileM + (C == 16 ? 4 : (C == 32 ? 2 : 1));
}

template <int CIN, int COUT, int XM, int YM>
__global__ void __launch_bounds__(kThreads) k_conv_wgrad(WgrArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int KCX = CIN / 8, KCY = COUT / 8;
    constexpr int RPD = dy_pitch<COUT>();
    constexpr uint32_t DB = (uint32_t)KCY * RPD * 16;
    const Geom g = a.g;
    const int tid = threadIdx.x;
    const int rows = stage_rows(g);
    const int RP = row_pitch(rows, CIN);
    const uint32_t SB = (uint32_t)KCX * RP * 16;
    const uint32_t RBX = XM == IN_EMBED ? raw_bytes(rows) : 0u;
    const uint32_t RBY = YM == IN_EMBED ? raw_bytes(kTileM) : 0u;
    uint8_t* dys = smem;
    uint8_t* xs = smem + 2 * DB;
    float* xraw = reinterpret_cast<float*>(xs + 4 * SB);
    float* yraw = reinterpret_cast<float*>(xs + 4 * SB + 4 * RBX);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(xs + 4 * SB + 4 * RBX + 2 * RBY);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);

    const int P0 = blockIdx.x * kTileM;
    const int I0 = 1 + blockIdx.y * a.ppc;
    const int t0 = blockIdx.z * a.tpg, t1 = min(kTaps, t0 + a.tpg);
    if (I0 > g.n0 || t0 >= kTaps) return;
    const int I1 = min(g.n0, I0 + a.ppc - 1);

    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_fence_init();
    }
    if (XM == IN_EMBED) stage_zero(xs, 4 * SB);
    if (YM == IN_EMBED) stage_zero(dys, 2 * DB);
    if (tid < 32) tmem_alloc(tslot, a.cols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;

    const int64_t pbase = (int64_t)P0 - g.W - 1;
    for (int I = I0 - 1; I <= I0 + 1; I++)
        stage<CIN, XM>(xs + (I & 3) * SB, xraw + (I & 3) * (RBX / 4), a.x, a.x32, g, (int64_t)I * g.plane + pbase,
                       rows, RP, rows);
    // dY only at the tile's positions inside this plane: on coarse levels a
    // 128-position tile runs past the plane's end into the next plane's rows,
    // which that plane's own pass counts
    const int yrows = min(kTileM, g.plane - P0);
    stage<COUT, YM>(dys + (I0 & 1) * DB, yraw + (I0 & 1) * (RBY / 4), a.dy, a.dy32, g, (int64_t)I0 * g.plane + P0,
                    kTileM, RPD, yrows);
    cp_commit();

    constexpr uint32_t idesc = idesc_bf16(kTileM, CIN, 1, 1);
    uint32_t phase = 0;
    bool aborted = false;
    for (int I = I0; I <= I1; I++) {
        const int buf = (I - I0) & 1;
        cp_wait_all();
        for (int p = (I == I0 ? I0 - 1 : I + 1); p <= I + 1; p++)
            stage_finish<XM>(xs + (p & 3) * SB, xraw + (p & 3) * (RBX / 4), rows);
        stage_finish<YM>(dys + (I & 1) * DB, yraw + (I & 1) * (RBY / 4), kTileM);
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
            const uint32_t xa = smem_u32(xs), ya = smem_u32(dys) + (I & 1) * DB;
#pragma unroll 1
            for (int t = t0; t < t1; t++) {
                const int di = t / 9 - 1, dj = (t / 3) % 3 - 1, dk = t % 3 - 1;
                const uint32_t xb = xa + ((I + di) & 3) * SB + (uint32_t)((dj + 1) * g.W + (dk + 1)) * 16;
                const uint32_t d = tmem + (uint32_t)(t - t0) * CIN;
#pragma unroll
                for (int s = 0; s < kTileM / 16; s++)
                    mma_bf16(d, smem_desc(ya + s * 256, 128, RPD * 16), smem_desc(xb + s * 256, 128, RP * 16), idesc,
                             (I == I0 && s == 0) ? 0u : 1u);
            }
            mma_commit(smem_u32(&mbar[buf]));
        }
        if (I > I0) {
            const int pb = buf ^ 1;
            const bool ok = mbar_wait(&mbar[pb], (phase >> pb) & 1u, a.err, 3);
            phase ^= 1u << pb;
            if (__syncthreads_or(!ok)) {
                aborted = true;
                break;
            }
        }
        if (I + 2 <= I1 + 1)
            stage<CIN, XM>(xs + ((I + 2) & 3) * SB, xraw + ((I + 2) & 3) * (RBX / 4), a.x, a.x32, g,
                           (int64_t)(I + 2) * g.plane + pbase, rows, RP, rows);
        if (I + 1 <= I1)
            stage<COUT, YM>(dys + ((I + 1) & 1) * DB, yraw + ((I + 1) & 1) * (RBY / 4), a.dy, a.dy32, g,
                            (int64_t)(I + 1) * g.plane + P0, kTileM, RPD, yrows);
        cp_commit();
    }
    if (!aborted) {
        const int lb = (I1 - I0) & 1;
        const bool ok = mbar_wait(&mbar[lb], (phase >> lb) & 1u, a.err, 4);
        if (!__syncthreads_or(!ok)) {
            fence_after_sync();
            const int warp = tid >> 5, lane = tid & 31;
            if (warp * 32 < COUT) {
                const int co = warp * 32 + lane;
                const int ncol = (t1 - t0) * CIN;
                const size_t cta = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
                float* base = a.part + cta * (size_t)a.tpg * COUT * CIN;
#pragma unroll 1
                for (int col = 0; col < ncol; col += 16) {
                    uint32_t r[16];
                    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + col, r);
                    tmem_wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; i++) reg_fence(r[i]);
                    if (co < COUT) {
                        const int tl = col / CIN, ci0 = col - tl * CIN;
                        float4* d = reinterpret_cast<float4*>(base + ((size_t)tl * COUT + co) * CIN + ci0);
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            d[i] = make_float4(__uint_as_float(r[4 * i]), __uint_as_float(r[4 * i + 1]),
                                               __uint_as_float(r[4 * i + 2]), __uint_as_float(r[4 * i + 3]));
                    }
                }
            }
        }
    }
    cp_wait_all();
    fence_before_sync();
    __syncthreads();
    if (tid < 32) {
        fence_after_sync();
        tmem_dealloc(tmem, a.cols);
    }
}

// grad[t][co][ci] += scale * sum over the CTAs of tap group t / tpg (fixed order)
__global__ void k_wgrad_reduce(const float* __restrict__ part, int nxy, int tpg, int CINK, int COUTK, int cin,
                               int cout, float scale, float* __restrict__ grad) {
    const int total = kTaps * cout * cin;
    const size_t ps = (size_t)tpg * COUTK * CINK;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        const int ci = idx % cin, co = (idx / cin) % cout, t = idx / (cin * cout);
        const int z = t / tpg, tl = t - z * tpg;
        const float* p = part + (size_t)z * nxy * ps + ((size_t)tl * COUTK + co) * CINK + ci;
        double s = 0.;
        for (int b = 0; b < nxy; b++) s += (double)p[(size_t)b * ps];
        grad[idx] += scale * (float)s;
    }
}

// ---------------------------------------------------------------------------
// level transfer: 2x2x2 restriction (scale 1/8 = average pool, 1 = the
// transpose of nearest prolongation) and the transpose of the average pool
// added into the finer level
template <int C>
__global__ void k_restrict(Geom f, Geom c, const bf16* __restrict__ fine, bf16* __restrict__ coarse, float scale) {
    constexpr int KC = C / 8;
    const int64_t total = (int64_t)c.n0 * c.n1 * c.n2 * KC;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int kc = (int)(idx % KC);
        int64_t v = idx / KC;
        const int k = (int)(v % c.n2);
        v /= c.n2;
        const int j = (int)(v % c.n1);
        const int i = (int)(v / c.n1);
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ch = 0; ch < 8; ch++) {
            const int fi = 2 * i + 1 + (ch >> 2), fj = 2 * j + 1 + ((ch >> 1) & 1), fk = 2 * k + 1 + (ch & 1);
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(
                fine + act_off(f.total, ((int64_t)fi * (f.n1 + 2) + fj) * f.W + fk, kc)));
            acc[0] += bf16_lo(q.x);
            acc[1] += bf16_hi(q.x);
            acc[2] += bf16_lo(q.y);
            acc[3] += bf16_hi(q.y);
            acc[4] += bf16_lo(q.z);
            acc[5] += bf16_hi(q.z);
            acc[6] += bf16_lo(q.w);
            acc[7] += bf16_hi(q.w);
        }
        uint4 o;
        o.x = pack_bf16(acc[0] * scale, acc[1] * scale);
        o.y = pack_bf16(acc[2] * scale, acc[3] * scale);
        o.z = pack_bf16(acc[4] * scale, acc[5] * scale);
        o.w = pack_bf16(acc[6] * scale, acc[7] * scale);
        *reinterpret_cast<uint4*>(coarse + act_off(c.total, ((int64_t)(i + 1) * (c.n1 + 2) + (j + 1)) * c.W + (k + 1), kc)) =
            o;
    }
}

// fine += scale * (nearest prolongation of coarse), one block per (chunk,
// i, j) line of fine cells, its threads along k
template <int C>
__global__ void k_prolong_add(Geom f, Geom c, const bf16* __restrict__ coarse, bf16* __restrict__ fine, float scale) {
    constexpr int KC = C / 8;
    const int lines = f.n0 * f.n1;
    for (int line = blockIdx.x; line < lines * KC; line += gridDim.x) {
        const int kc = line / lines;
        const int ij = line - kc * lines;
        const int i = ij / f.n1, j = ij - (ij / f.n1) * f.n1;
        const int64_t fq = ((int64_t)(i + 1) * (f.n1 + 2) + (j + 1)) * f.W + 1;
        const int64_t cq = ((int64_t)(i / 2 + 1) * (c.n1 + 2) + (j / 2 + 1)) * c.W + 1;
        for (int k = threadIdx.x; k < f.n2; k += blockDim.x) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(coarse + act_off(c.total, cq + k / 2, kc)));
            uint4* dst = reinterpret_cast<uint4*>(fine + act_off(f.total, fq + k, kc));
            const uint4 o = *dst;
            uint4 r;
            r.x = pack_bf16(bf16_lo(o.x) + scale * bf16_lo(q.x), bf16_hi(o.x) + scale * bf16_hi(q.x));
            r.y = pack_bf16(bf16_lo(o.y) + scale * bf16_lo(q.y), bf16_hi(o.y) + scale * bf16_hi(q.y));
            r.z = pack_bf16(bf16_lo(o.z) + scale * bf16_lo(q.z), bf16_hi(o.z) + scale * bf16_hi(q.z));
            r.w = pack_bf16(bf16_lo(o.w) + scale * bf16_lo(q.w), bf16_hi(o.w) + scale * bf16_hi(q.w));
            *dst = r;
        }
    }
}

// padded bf16 activations -> FP32 [cell][C] over the internal cells
__global__ void k_read_act(Geom g, int C, const bf16* __restrict__ a, float* __restrict__ out) {
    const int64_t total = (int64_t)g.n0 * g.n1 * g.n2 * C;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(idx % C);
        int64_t v = idx / C;
        const int k = (int)(v % g.n2);
        v /= g.n2;
        const int j = (int)(v % g.n1);
        const int i = (int)(v / g.n1);
        out[idx] = __bfloat162float(
            a[act_off(g.total, ((int64_t)(i + 1) * (g.n1 + 2) + (j + 1)) * g.W + (k + 1), ch / 8) + ch % 8]);
    }
}

// ---------------------------------------------------------------------------
// loss: w = scale / ||e||^2; g = 2 w (z - e); loss += w ||z - e||^2
__global__ void __launch_bounds__(256) k_loss_grad(int64_t n, const float* __restrict__ z, const float* __restrict__ e,
                                                   const float* __restrict__ en2, float scale, float* __restrict__ g,
                                                   double* __restrict__ loss) {
    __shared__ double sh[8];
    const float w = scale / fmaxf(*en2, 1e-30f);
    double acc = 0.;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const float d = z[c] - e[c];
        g[c] = 2.f * w * d;
        acc += (double)d * d;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
        atomicAdd(loss, s * (double)w);
    }
}

__global__ void k_adam(int64_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// master weights [27][cout][cin] -> packed bf16 [nz][9 (di,dj)][CINK/8][3 dk][NT][8]
// (the B operand of k_conv_fwd: for one (di, dj) and K chunk, N rows dk NT + n).
// flip: the data-gradient convolution (input cout channels, output cin),
// W'[t][o][i] = W[26 - t][i][o].
__global__ void k_pack(const float* __restrict__ W, int cin, int cout, int CINK, int NT, int nz, int flip,
                       bf16* __restrict__ out) {
    const int KC = CINK / 8;
    const int64_t total = (int64_t)nz * kTaps * KC * NT * 8;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = idx;
        const int e = (int)(r % 8);
        r /= 8;
        const int n = (int)(r % NT);
        r /= NT;
        const int dk = (int)(r % 3);
        r /= 3;
        const int kc = (int)(r % KC);
        r /= KC;
        const int g9 = (int)(r % 9);
        const int z = (int)(r / 9);
        const int t = 3 * g9 + dk;
        const int o = z * NT + n, i = kc * 8 + e;
        float v = 0.f;
        if (!flip) {
            if (o < cout && i < cin) v = W[((int64_t)t * cout + o) * cin + i];
        } else {
            if (o < cin && i < cout) v = W[((int64_t)(kTaps - 1 - t) * cout + i) * cin + o];
        }
        out[idx] = __float2bfloat16_rn(v);
    }
}

// One-channel-input weights for the window rows of k_conv_in, the di taps
// along N: out[c][16 di + n][e] = W(t, n) with, for e < 6, dj = 2 c + e / 3,
// dk = e % 3, t = 9 di + 3 dj + dk when dj < 3; 0 otherwise.
// W(t, n) = W[t][n][0] (enc0, cout 16, cin 1) or, flipped for the dec0 data
// gradient, W[26 - t][0][n] (cout 1, cin 16).
__global__ void k_pack_tapk(const float* __restrict__ W, int flip, bf16* __restrict__ out) {
    for (int idx = threadIdx.x; idx < 2 * 48 * 8; idx += blockDim.x) {
        const int e = idx & 7, nn = (idx >> 3) % 48, c = idx / (8 * 48);
        const int di = nn / 16, n = nn - 16 * (nn / 16);
        const int dj = 2 * c + e / 3, dk = e - 3 * (e / 3);
        float v = 0.f;
        if (e < 6 && dj < 3) {
            const int t = di * 9 + dj * 3 + dk;
            v = flip ? W[(kTaps - 1 - t) * 16 + n] : W[t * 16 + n];
        }
        out[idx] = __float2bfloat16_rn(v);
    }
}

// dec0 forward weights, (di, dk) along N: out[dj][kc][n][e] = W[t][0][8 kc + e]
// with t = 9 di + 3 dj + dk for n = 3 di + dk < 9, else 0.
__global__ void k_pack_tapn(const float* __restrict__ W, bf16* __restrict__ out) {
    for (int idx = threadIdx.x; idx < 3 * 2 * 16 * 8; idx += blockDim.x) {
        const int e = idx & 7, n = (idx >> 3) & 15, kc = (idx >> 7) & 1, dj = idx >> 8;
        const int di = n / 3, dk = n - 3 * (n / 3);
        out[idx] = __float2bfloat16_rn(n < 9 ? W[(9 * di + 3 * dj + dk) * 16 + kc * 8 + e] : 0.f);
    }
}

// ---------------------------------------------------------------------------
// pair generation: r = b - A x_k (FP32), e = diag_C (x* - x_k) (FP32),
// acc += ||e||^2 (FP64, atomically)
__global__ void __launch_bounds__(256) k_make_pair(GridDev g, const double* __restrict__ diag,
                                                   const double* __restrict__ b, const double* __restrict__ xk,
                                                   const double* __restrict__ xs, float* __restrict__ r,
                                                   float* __restrict__ e, double* __restrict__ acc) {
    __shared__ double sh[8];
    const int64_t n = g.ncell, nyz = (int64_t)g.n[1] * g.n[2];
    double s = 0.;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c / nyz), j = (int)((c / g.n[2]) % g.n[1]), k = (int)(c % g.n[2]);
        int64_t nb[7];
        neighbour_ordinals(g, i, j, k, c, nb);
        double ax = 0.;
#pragma unroll
        for (int q = 0; q < 7; q++) ax += diag[q * n + c] * xk[nb[q]];
        r[c] = (float)(b[c] - ax);
        const float ev = (float)(diag[c] * (xs[c] - xk[c]));
        e[c] = ev;
        s += (double)ev * ev;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        atomicAdd(acc, t);
    }
}

__global__ void k_store_norm(const double* acc, float* out) { *out = (float)*acc; }

__global__ void __launch_bounds__(256) k_sqnorm(int64_t n, const float* __restrict__ e, double* __restrict__ acc) {
    __shared__ double sh[8];
    double s = 0.;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        s += (double)e[c] * e[c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        atomicAdd(acc, t);
    }
}

// y = D x: the right-preconditioned solve iterates on y with x = D^-1 y and
// takes its initial guess as y0 (BiCGStab2.inl:258-261 with the Jacobi
// preconditioner), so a warm start at the physical x passes D x
__global__ void k_warm(int64_t n, const double* __restrict__ diag, const double* __restrict__ x, double* __restrict__ y) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        y[c] = diag[c] * x[c];
}

// ---------------------------------------------------------------------------
// coarse-correction form: level transfers between the system's grid (2 c0,
// 2 c1, 2 c2) and the network's grid (c0, c1, c2), FP32, cell layout.
// uc = R u: the mean of the 8 children.  A thread makes two neighbouring
// coarse cells (K = 2 K2, 2 K2 + 1) from four 16-byte loads of fine rows
// (the coarse sizes are multiples of 8, so rows split into whole pairs).
__global__ void __launch_bounds__(256) k_pool8(int c0, int c1, int c2, const float* __restrict__ f,
                                               float* __restrict__ c) {
    const int h2 = c2 / 2;
    const int64_t nq = (int64_t)c0 * c1 * h2;
    const int64_t F2 = 2 * (int64_t)c2, F1 = 2 * (int64_t)c1;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t K2 = q % h2, JI = q / h2, J = JI % c1, I = JI / c1;
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const float4 v = *reinterpret_cast<const float4*>(f + ((2 * I + a) * F1 + 2 * J + b) * F2 + 4 * K2);
                s0 += v.x + v.y;
                s1 += v.z + v.w;
            }
        *reinterpret_cast<float2*>(c + JI * c2 + 2 * K2) = make_float2(0.125f * s0, 0.125f * s1);
    }
}

// z = u + P (zc - uc): every fine cell adds its parent's network correction;
// a thread handles four fine cells along k (two parents) with 16-byte
// accesses
__global__ void __launch_bounds__(256) k_coarse_add(int c0, int c1, int c2, const float* __restrict__ u,
                                                    const float* __restrict__ zc, const float* __restrict__ uc,
                                                    float* __restrict__ z) {
    const int h2 = c2 / 2;
    const int64_t F2 = 2 * (int64_t)c2, F1 = 2 * (int64_t)c1;
    const int64_t nq = (int64_t)2 * c0 * F1 * h2;   // fine cells / 4
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t K2 = q % h2, row = q / h2;          // row = fine (i, j)
        const int64_t j = row % F1, i = row / F1;
        const int64_t p = ((i >> 1) * c1 + (j >> 1)) * c2 + 2 * K2;
        const float2 zz = *reinterpret_cast<const float2*>(zc + p), uu = *reinterpret_cast<const float2*>(uc + p);
        const float d0 = zz.x - uu.x, d1 = zz.y - uu.y;
        const float4 v = *reinterpret_cast<const float4*>(u + row * F2 + 4 * K2);
        *reinterpret_cast<float4*>(z + row * F2 + 4 * K2) = make_float4(v.x + d0, v.y + d0, v.z + d1, v.w + d1);
    }
}

// ---------------------------------------------------------------------------
// host side: launch configuration and dispatch
static size_t fwd_smem(int cin, int nt, const Geom& g, int mt, int slots) {
    const int RP = round8(strip_rows(g, mt));
    return (size_t)kTaps * cin * nt * 2 + slots * (size_t)(cin / 8) * RP * 16 + 2 * (size_t)mt * 4 * 2 * nt * 4 +
           (2 * kMaxSlots + 5) * 8 + 16;
}

// two M tiles per step on planes wider than two tiles, when a 4-slot ring of
// the wider plane segments still fits
// M tiles per CTA of k_conv_fwd: one tile when that at least doubles the CTAs
// an SM holds (shared memory with the shallowest ring, TMEM columns), two
// otherwise (fewer halo rows per output).  A CTA's loop over its planes is
// latency-bound, so CTAs per SM count more than rows per CTA (enc1 at 256^3:
// 116 us with two tiles at one CTA per SM, 96 us with one tile at two).
static int pick_mt(const Geom& g, int cin, int nt) {
    auto occ = [&](int mt) -> int {
        const size_t smem = fwd_smem(cin, nt, g, mt, 4);
        if (smem > kMaxSmem) return 0;
        const uint32_t acols = 2 * mt * (3 * nt <= 64 ? 64 : 128);
        const uint32_t cols = acols <= 128 ? 128 : (acols <= 256 ? 256 : 512);
        return (int)std::min<size_t>(233472 / (smem + 1024), 512 / cols);
    };
    if (g.plane <= 2 * kOutStride) return 1;
    const int o1 = occ(1), o2 = occ(2);
    return o2 > 0 && o1 < 2 * o2 ? 2 : 1;
}

// Planes per CTA of a plane-marching grid with `units` CTAs per chunk of
// planes: the choice that minimises the modelled time waves x (planes + 3)
// (a CTA stages two planes more than it computes, plus its set-up), waves =
// ceil(units x chunks / resident CTAs).
static int pick_ppc(int n0, int64_t units, int64_t resident) {
    int best = n0;
    int64_t best_cost = INT64_MAX;
    for (int chunks = 1; chunks <= n0; chunks++) {
        const int ppc = (n0 + chunks - 1) / chunks;
        if ((n0 + ppc - 1) / ppc != chunks) continue;
        const int64_t waves = (units * chunks + resident - 1) / resident;
        const int64_t cost = waves * (ppc + 3);
        if (cost < best_cost) {
            best_cost = cost;
            best = ppc;
        }
    }
    return best;
}

static int dy_pitch_rt(int c) { return kTileM + (c == 16 ? 4 : (c == 32 ? 2 : 1)); }

static size_t wgr_smem(int cin, int cout, const Geom& g, bool xembed, bool yembed) {
    const int rows = stage_rows(g);
    const int RP = row_pitch(rows, cin);
    const size_t DB = (size_t)(cout / 8) * dy_pitch_rt(cout) * 16;
    const size_t body = 2 * DB + 4 * (size_t)(cin / 8) * RP * 16 + (xembed ? 4 * (size_t)raw_bytes(rows) : 0) +
                        (yembed ? 2 * (size_t)raw_bytes(kTileM) : 0) + 32;
    // the A operand (dY^T, 128 rows of which Cout are real) of the second dY
    // slot reaches 16 row groups past its start: keep that inside the CTA
    const size_t reach = DB + (size_t)(kTileM / 16) * 256 + 15 * (size_t)dy_pitch_rt(cout) * 16 + 256;
    return std::max(body, reach + 32);
}

template <typename K>
static int occupancy_fit(dare_ctx* ctx, K kern, size_t& smem, uint32_t cols, int* occ_out,
                         int threads = kThreads) {
    DARE_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    DARE_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
    // Resident CTAs per SM from the kernel's registers, threads and shared
    // memory (the runtime's occupancy query answers 1 for these kernels,
    // while the hardware keeps as many as the resources allow).
    cudaFuncAttributes fa;
    DARE_CUDA(ctx, cudaFuncGetAttributes(&fa, kern));
    const int warps = (threads + 31) / 32;
    const int regs_warp = ((fa.numRegs + 7) / 8) * 8 * 32;
    const int by_regs = 65536 / (warps * ((regs_warp + 255) / 256) * 256);
    const int by_threads = 2048 / (warps * 32);
    int occ = 0;
    for (;;) {
        const int by_smem = (int)(233472 / (smem + fa.sharedSizeBytes + 1024));
        occ = std::min(std::min(by_regs, by_threads), std::min(by_smem, 32));
        // CTAs resident on one SM must never ask for more than its 512 TMEM columns
        if (occ * cols <= 512 || smem + 4096 > kMaxSmem) break;
        smem += 4096;
    }
    if (occ < 1 || occ * cols > 512) return set_error(ctx, DARE_ERR_UNSUPPORTED, "unet: no launchable configuration");
    *occ_out = occ;
    return DARE_OK;
}

template <int CIN, int NT, int MT, int OUTM>
static int launch_fwd_t(dare_ctx* ctx, LaunchCfg& lc, int nz, const FwdArgs& a0) {
    auto kern = k_conv_fwd<CIN, NT, MT, OUTM>;
    if (!lc.ready) {
        const uint32_t acols = 2 * MT * (3 * NT <= 64 ? 64 : 128);
        const uint32_t cols = acols <= 128 ? 128 : (acols <= 256 ? 256 : 512);
        const int slots = pick_slots([&](int sl) { return fwd_smem(CIN, NT, a0.g, MT, sl); }, cols);
        size_t smem = fwd_smem(CIN, NT, a0.g, MT, slots);
        if (smem > kMaxSmem) return set_error(ctx, DARE_ERR_UNSUPPORTED, "unet: level too wide for the staged conv");
        int occ = 0, rc;
        if ((rc = occupancy_fit(ctx, kern, smem, cols, &occ, fwd_threads(MT)))) return rc;
        const int n0 = a0.g.n0;
        const int tiles = (a0.g.plane + MT * kOutStride - 1) / (MT * kOutStride);
        const int ppc = pick_ppc(n0, (int64_t)tiles * nz, (int64_t)ctx->num_sms * occ);
        lc.ppc = ppc;
        lc.occ = occ;
        lc.mt = MT;
        lc.slots = slots;
        lc.grid = dim3(tiles, (n0 + ppc - 1) / ppc, nz);
        lc.smem = smem;
        lc.cols = cols;
        lc.ready = true;
    }
    FwdArgs a = a0;
    a.ppc = lc.ppc;
    a.slots = lc.slots;
    kern<<<lc.grid, fwd_threads(MT), lc.smem, ctx->stream>>>(a);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// BF16 input `a.in` with `cin` channels
static int launch_fwd(dare_ctx* ctx, LaunchCfg& lc, int cin, int nt, int nz, int outm, const FwdArgs& a) {
    const int mt = pick_mt(a.g, cin, nt);
#define DARE_FWD(CI, N, OM)                                                                       \
    if (cin == CI && nt == N && outm == OM)                                                       \
        return mt == 2 ? launch_fwd_t<CI, N, 2, OM>(ctx, lc, nz, a) : launch_fwd_t<CI, N, 1, OM>(ctx, lc, nz, a);
    DARE_FWD(16, 16, OUT_STORE)
    DARE_FWD(16, 32, OUT_STORE)
    DARE_FWD(32, 16, OUT_STORE)
    DARE_FWD(32, 32, OUT_STORE)
    DARE_FWD(64, 16, OUT_STORE)
    DARE_FWD(64, 32, OUT_STORE)
    DARE_FWD(32, 16, OUT_ADDUP)
    DARE_FWD(64, 16, OUT_ADDUP)
    DARE_FWD(64, 32, OUT_ADDUP)
#undef DARE_FWD
    return set_error(ctx, DARE_ERR_UNSUPPORTED, "unet: no forward convolution kernel for this shape");
}

template <int CIN, int COUT, int XM, int YM>
static int launch_wgr_t(dare_ctx* ctx, LaunchCfg& lc, WgrArgs a, size_t* part_need) {
    auto kern = k_conv_wgrad<CIN, COUT, XM, YM>;
    if (!lc.ready) {
        size_t smem = wgr_smem(CIN, COUT, a.g, XM == IN_EMBED, YM == IN_EMBED);
        if (smem > kMaxSmem) return set_error(ctx, DARE_ERR_UNSUPPORTED, "unet: level too wide for the staged conv");
        const int tpg = std::min(kTaps, 256 / CIN);
        uint32_t cols = 32;
        while (cols < (uint32_t)(tpg * CIN)) cols <<= 1;
        int occ = 0, rc;
        if ((rc = occupancy_fit(ctx, kern, smem, cols, &occ))) return rc;
        const int groups = (kTaps + tpg - 1) / tpg;
        const int n0 = a.g.n0;
        const int64_t target = (int64_t)ctx->num_sms * occ * 2;
        const int64_t per = (int64_t)a.g.tiles * groups;
        int chunks = (int)std::min<int64_t>(n0, std::max<int64_t>(1, (target + per - 1) / per));
        const int ppc = (n0 + chunks - 1) / chunks;
        lc.ppc = ppc;
        lc.tpg = tpg;
        lc.cols = cols;
        lc.occ = occ;
        lc.grid = dim3(a.g.tiles, (n0 + ppc - 1) / ppc, groups);
        lc.smem = smem;
        lc.ready = true;
    }
    *part_need = (size_t)lc.grid.x * lc.grid.y * lc.grid.z * lc.tpg * COUT * CIN;
    if (!a.part) return DARE_OK;  // sizing pass
    a.ppc = lc.ppc;
    a.tpg = lc.tpg;
    a.cols = lc.cols;
    kern<<<lc.grid, kThreads, lc.smem, ctx->stream>>>(a);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

static int launch_wgr(dare_ctx* ctx, LaunchCfg& lc, int cin, int cout, int xm, int ym, const WgrArgs& a,
                      size_t* part_need) {
#define DARE_WGR(CI, CO, XM, YM) \
    if (cin == CI && cout == CO && xm == XM && ym == YM) return launch_wgr_t<CI, CO, XM, YM>(ctx, lc, a, part_need);
    DARE_WGR(16, 16, IN_EMBED, IN_BF16)
    DARE_WGR(16, 32, IN_BF16, IN_BF16)
    DARE_WGR(32, 64, IN_BF16, IN_BF16)
    DARE_WGR(64, 64, IN_BF16, IN_BF16)
    DARE_WGR(64, 32, IN_BF16, IN_BF16)
    DARE_WGR(32, 16, IN_BF16, IN_BF16)
    DARE_WGR(16, 16, IN_BF16, IN_EMBED)
#undef DARE_WGR
    return set_error(ctx, DARE_ERR_UNSUPPORTED, "unet: no weight-gradient kernel for this shape");
}

// Ring depth (4..8 staged planes) of a plane-marching kernel: the deepest ring
// among those that give the most resident CTAs per SM (shared memory of the
// SM, 228 KB, with 1 KB reserved per CTA; TMEM columns), so that short rings
// buy a second or third CTA where one deep ring would fill the SM.
template <typename SmemFn>
static int pick_slots(SmemFn smem_of, uint32_t cols) {
    constexpr size_t kSmemPerSM = 233472;
    int best = 0, best_occ = 0;
    for (int slots = 4; slots <= kMaxSlots; slots++) {
        const size_t smem = smem_of(slots);
        if (smem > kMaxSmem) break;
        const int occ = (int)std::min<size_t>(kSmemPerSM / (smem + 1024), 512 / cols);
        if (occ >= best_occ) {
            best_occ = occ;
            best = slots;
        }
    }
    return best > 0 ? best : 4;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on the driver library); no interleave, no swizzle,
// cells outside the tensor read zero.
static int encode_tiled(dare_ctx* ctx, CUtensorMap* m, CUtensorMapDataType type, int rank, const void* base,
                        const cuuint64_t* dims, const cuuint64_t* strides, const cuuint32_t* box, const cuuint32_t* es) {
    // looked up once (a function-local static is initialised thread-safely)
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return set_error(ctx, DARE_ERR_CUDA, "unet: cuTensorMapEncodeTiled is not available");
    const CUresult r = encode(m, type, (cuuint32_t)rank, const_cast<void*>(base), dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(ctx, DARE_ERR_CUDA, "unet: cuTensorMapEncodeTiled failed");
    return DARE_OK;
}

// tcgen05 tile count of k_conv_in per CTA (16 rows j each)
constexpr int kInMT = 1;

template <int MT>
static int launch_in_t(dare_ctx* ctx, LaunchCfg& lc, InArgs& a) {
    auto kern = k_conv_in<MT>;
    if (!lc.ready) {
        const uint32_t cols = kInAcc * kInB * MT * 64;
        size_t smem = in_smem(MT);
        int occ = 0, rc;
        if ((rc = occupancy_fit(ctx, kern, smem, cols, &occ, in_threads()))) return rc;
        const Geom& g = a.g;
        const int tiles = ((g.n2 + 7) / 8) * ((g.n1 + 16 * MT - 1) / (16 * MT));
        const int ppc0 = pick_ppc(g.n0, tiles, (int64_t)ctx->num_sms * occ);
        const int ppc = ppc0 + (ppc0 & 1);  // pairs of output planes stay in one CTA (n0 is even)
        lc.ppc = ppc;
        lc.occ = occ;
        lc.mt = MT;
        lc.slots = kInRaw;
        lc.grid = dim3(tiles, (g.n0 + ppc - 1) / ppc, 1);
        lc.smem = smem;
        lc.cols = cols;
        lc.ready = true;
    }
    a.ppc = lc.ppc;
    kern<<<lc.grid, in_threads(), lc.smem, ctx->stream>>>(a);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// The kernel reads in32 (FP32 over the internal cells) through a TMA map;
// a row pitch that is not a multiple of 16 bytes (n2 % 4 != 0) or a base
// that is not 16-byte aligned goes through a pitched copy in `stage` first.
static int launch_in(dare_ctx* ctx, LaunchCfg& lc, InArgs& a, const float* in32, float* stage) {
    const Geom& g = a.g;
    const float* base = in32;
    int64_t pitch = g.n2;
    if ((g.n2 & 3) || (reinterpret_cast<uintptr_t>(in32) & 15)) {
        pitch = (g.n2 + 3) & ~3;
        DARE_CUDA(ctx, cudaMemcpy2DAsync(stage, (size_t)pitch * 4, in32, (size_t)g.n2 * 4, (size_t)g.n2 * 4,
                                         (size_t)g.n0 * g.n1, cudaMemcpyDeviceToDevice, ctx->stream));
        base = stage;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g.n2, (cuuint64_t)g.n1, (cuuint64_t)g.n0};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * g.n1 * 4};
    const cuuint32_t box[3] = {(cuuint32_t)kInBoxK, (cuuint32_t)(16 * kInMT + 3), (cuuint32_t)kInB};
    const cuuint32_t es[3] = {1, 1, 1};
    int rc;
    if ((rc = encode_tiled(ctx, &a.x, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, es))) return rc;
    return launch_in_t<kInMT>(ctx, lc, a);
}

// shared memory of k_conv_out with `slots` staged groups of kOutB planes
static size_t out_smem(const Geom& g, int mt, int slots) {
    const int RP = round8(strip_rows(g, mt));
    return 3 * 2 * 16 * 16 + slots * (size_t)kOutB * 2 * RP * 16 + 2 * (size_t)mt * kTileM * 3 * 4 +
           (2 * kMaxSlots + 2 * kOutG + 1) * 8 + 16;
}

// staged groups: the most CTAs per SM, then the deepest ring (2 .. 8 groups)
static int out_slots(const Geom& g, int mt, uint32_t cols) {
    constexpr size_t kSmemPerSM = 233472;
    int best = 2, best_occ = 0;
    for (int sl = 2; sl <= kMaxSlots; sl++) {
        const size_t smem = out_smem(g, mt, sl);
        if (smem > kMaxSmem) break;
        const int occ = (int)std::min<size_t>(kSmemPerSM / (smem + 1024), 512 / cols);
        if (occ >= best_occ) {
            best_occ = occ;
            best = sl;
        }
    }
    return best;
}

static int out_tiles_mt(const Geom& g) {
    return g.plane > 2 * kOutStride && out_smem(g, 2, 2) <= kMaxSmem ? 2 : 1;
}

template <int MT>
static int launch_out_t(dare_ctx* ctx, LaunchCfg& lc, const OutArgs& a0) {
    auto kern = k_conv_out<MT>;
    if (!lc.ready) {
        const uint32_t cols = kOutG * kOutB * MT * 16 <= 64 ? 64 : 128;
        const int slots = out_slots(a0.g, MT, cols);
        size_t smem = out_smem(a0.g, MT, slots);
        if (smem > kMaxSmem) return set_error(ctx, DARE_ERR_UNSUPPORTED, "unet: level too wide for the staged conv");
        int occ = 0, rc;
        if ((rc = occupancy_fit(ctx, kern, smem, cols, &occ, out_threads(MT)))) return rc;
        const int n0 = a0.g.n0;
        const int tiles = (a0.g.plane + MT * kOutStride - 1) / (MT * kOutStride);
        const int ppc = pick_ppc(n0, tiles, (int64_t)ctx->num_sms * occ);
        lc.ppc = ppc;
        lc.occ = occ;
        lc.mt = MT;
        lc.slots = slots;
        lc.grid = dim3(tiles, (n0 + ppc - 1) / ppc, 1);
        lc.smem = smem;
        lc.cols = cols;
        lc.ready = true;
    }
    OutArgs a = a0;
    a.ppc = lc.ppc;
    a.slots = lc.slots;
    kern<<<lc.grid, out_threads(MT), lc.smem, ctx->stream>>>(a);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

static int launch_out(dare_ctx* ctx, LaunchCfg& lc, const OutArgs& a) {
    return out_tiles_mt(a.g) == 2 ? launch_out_t<2>(ctx, lc, a) : launch_out_t<1>(ctx, lc, a);
}

static int pick_nt(int cink, int coutk, const Geom& g) {
    if (coutk % 32 == 0 && fwd_smem(cink, 32, g, 1, 4) <= kMaxSmem) return 32;
    return 16;
}

static inline int eblocks(const dare_ctx* ctx, int64_t work) { return grid_blocks(ctx, work, 256, 8); }

// ---- network passes ----------------------------------------------------------
static int conv_forward(dare_unet* net, int l, const bf16* in, const float* in32, int outm, bf16* out, bf16* fine,
                        float* out32, const float* res32) {
    Layer& L = net->layer[l];
    if (l == ENC0) {
        InArgs a{};
        a.g = net->geo[0];
        a.w = L.wf;
        a.out = out;
        a.pool = net->P1;  // the average pool to level 1 rides on the epilogue
        a.cg = net->geo[1];
        a.pool_scale = 0.125f;
        a.err = net->err;
        a.wait_limit = net->wait_limit;
        return launch_in(net->ctx, L.fwd, a, in32, net->X0);
    }
    if (l == DEC0) {
        OutArgs a{};
        a.g = net->geo[0];
        a.in = in;
        a.w = L.wf;
        a.out32 = out32;
        a.res32 = res32;
        a.err = net->err;
        a.wait_limit = net->wait_limit;
        return launch_out(net->ctx, L.fwd, a);
    }
    FwdArgs a{};
    a.g = net->geo[L.level];
    if (L.level > 0) a.fg = net->geo[L.level - 1];
    a.in = in;
    a.w = L.wf;
    a.cout = L.coutk;
    a.out = out;
    a.fine = fine;
    a.err = net->err;
    a.wait_limit = net->wait_limit;
    a.skip_plane = net->debug_skip;   // one-shot test hook
    net->debug_skip = 0;
    return launch_fwd(net->ctx, L.fwd, L.cink, L.nt, L.coutk / L.nt, outm, a);
}

// data gradient of layer l: dX = conv(dY, W flipped and transposed)
static int conv_dgrad(dare_unet* net, int l, const bf16* dy, const float* dy32, bf16* dx) {
    Layer& L = net->layer[l];
    if (l == DEC0) {
        InArgs a{};
        a.g = net->geo[0];
        a.w = L.wb;
        a.out = dx;
        a.pool = net->dD1;  // the restriction (sum) to level 1, transposing the prolongation
        a.cg = net->geo[1];
        a.pool_scale = 1.f;
        a.err = net->err;
        a.wait_limit = net->wait_limit;
        return launch_in(net->ctx, L.bwd, a, dy32, net->X0);
    }
    FwdArgs a{};
    a.g = net->geo[L.level];
    a.in = dy;
    a.w = L.wb;
    a.cout = L.cink;
    a.out = dx;
    a.err = net->err;
    a.wait_limit = net->wait_limit;
    return launch_fwd(net->ctx, L.bwd, L.coutk, L.ntb, L.cink / L.ntb, OUT_STORE, a);
}

static int conv_wgrad(dare_unet* net, int l, const bf16* x, const float* x32, const bf16* dy, const float* dy32,
                      float scale) {
    Layer& L = net->layer[l];
    dare_ctx* ctx = net->ctx;
    WgrArgs a{};
    a.g = net->geo[L.level];
    a.x = x;
    a.x32 = x32;
    a.dy = dy;
    a.dy32 = dy32;
    a.err = net->err;
    size_t need = 0;
    int rc = launch_wgr(ctx, L.wgr, L.cink, L.coutk, x32 ? IN_EMBED : IN_BF16, dy32 ? IN_EMBED : IN_BF16, a, &need);
    if (rc) return rc;
    if (need > net->part_floats) {
        cudaFree(net->part);
        net->part = nullptr;
        net->part_floats = 0;
        DARE_CUDA(ctx, cudaMalloc(&net->part, need * sizeof(float)));
        net->part_floats = need;
    }
    a.part = net->part;
    if ((rc = launch_wgr(ctx, L.wgr, L.cink, L.coutk, x32 ? IN_EMBED : IN_BF16, dy32 ? IN_EMBED : IN_BF16, a, &need)))
        return rc;
    const int nxy = (int)(L.wgr.grid.x * L.wgr.grid.y);
    k_wgrad_reduce<<<eblocks(ctx, kTaps * L.cin * L.cout), 256, 0, ctx->stream>>>(
        net->part, nxy, L.wgr.tpg, L.cink, L.coutk, L.cin, L.cout, scale, net->grad + L.woff);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

template <int C>
static int restrict_to(dare_unet* net, int fl, const bf16* fine, bf16* coarse, float scale) {
    dare_ctx* ctx = net->ctx;
    const Geom& c = net->geo[fl + 1];
    k_restrict<C><<<eblocks(ctx, (int64_t)c.n0 * c.n1 * c.n2 * (C / 8)), 256, 0, ctx->stream>>>(net->geo[fl], c, fine,
                                                                                                coarse, scale);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

template <int C>
static int prolong_add(dare_unet* net, int fl, const bf16* coarse, bf16* fine, float scale) {
    dare_ctx* ctx = net->ctx;
    const Geom& f = net->geo[fl];
    const int64_t lines = (int64_t)f.n0 * f.n1 * (C / 8);
    k_prolong_add<C><<<(int)std::min<int64_t>(lines, (int64_t)ctx->num_sms * 16), 128, 0, ctx->stream>>>(
        f, net->geo[fl + 1], coarse, fine, scale);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// z = u + U(u) on the network's own grid
static int apply_grid(dare_unet* net, const float* u, float* z) {
    int rc;
    // enc0 also writes P1, the average pool of S0
    if ((rc = conv_forward(net, ENC0, nullptr, u, OUT_STORE, net->S0, nullptr, nullptr, nullptr))) return rc;
    if ((rc = conv_forward(net, ENC1, net->P1, nullptr, OUT_STORE, net->S1, nullptr, nullptr, nullptr))) return rc;
    if ((rc = restrict_to<32>(net, 1, net->S1, net->P2, 0.125f))) return rc;
    if ((rc = conv_forward(net, ENC2, net->P2, nullptr, OUT_STORE, net->S2, nullptr, nullptr, nullptr))) return rc;
    if ((rc = restrict_to<64>(net, 2, net->S2, net->P3, 0.125f))) return rc;
    if ((rc = conv_forward(net, ENC3, net->P3, nullptr, OUT_STORE, net->E3, nullptr, nullptr, nullptr))) return rc;
    if ((rc = conv_forward(net, DEC3, net->E3, nullptr, OUT_ADDUP, nullptr, net->S2, nullptr, nullptr))) return rc;
    if ((rc = conv_forward(net, DEC2, net->S2, nullptr, OUT_ADDUP, nullptr, net->S1, nullptr, nullptr))) return rc;
    // dec1 stores its level-1 output (into dD1, free during the forward pass)
    // and a streaming pass adds its prolongation into S0: that read-modify-
    // write of S0 inside the convolution's epilogue was latency-bound
    if ((rc = conv_forward(net, DEC1, net->S1, nullptr, OUT_STORE, net->dD1, nullptr, nullptr, nullptr))) return rc;
    if ((rc = prolong_add<16>(net, 0, net->dD1, net->S0, 1.f))) return rc;
    return conv_forward(net, DEC0, net->S0, nullptr, OUT_F32, nullptr, nullptr, z, u);
}

int apply(dare_unet* net, const float* u, float* z) {
    if (!net->coarse) return apply_grid(net, u, z);
    // coarse form: z = u + P (N_c(R u) - R u), N_c(v) = v + U(v) on the coarse grid
    dare_ctx* ctx = net->ctx;
    float* uc = net->cbuf;
    float* zc = net->cbuf + net->ncell;
    // (16-byte accesses: u and z must be 16-byte aligned; an unaligned
    // caller vector is copied first)
    const float* uin = u;
    float* zout = z;
    if ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(z)) & 15) {
        if (!net->fbuf) DARE_CUDA(ctx, cudaMalloc(&net->fbuf, (size_t)2 * net->fine_ncell * sizeof(float)));
        DARE_CUDA(ctx, cudaMemcpyAsync(net->fbuf, u, net->fine_ncell * sizeof(float), cudaMemcpyDeviceToDevice,
                                       ctx->stream));
        uin = net->fbuf;
        zout = net->fbuf + net->fine_ncell;
    }
    k_pool8<<<eblocks(ctx, net->ncell / 2), 256, 0, ctx->stream>>>(net->n[0], net->n[1], net->n[2], uin, uc);
    DARE_LAUNCHED(ctx);
    int rc = apply_grid(net, uc, zc);
    if (rc) return rc;
    k_coarse_add<<<eblocks(ctx, net->fine_ncell / 4), 256, 0, ctx->stream>>>(net->n[0], net->n[1], net->n[2], uin, zc,
                                                                              uc, zout);
    DARE_LAUNCHED(ctx);
    if (zout != z)
        DARE_CUDA(ctx, cudaMemcpyAsync(z, zout, net->fine_ncell * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

// Backward pass of the last apply() for input u and output gradient g;
// adds scale * dL/dW to net->grad.
static int backward(dare_unet* net, const float* u, const float* g, float scale) {
    int rc;
    if ((rc = conv_wgrad(net, DEC0, net->S0, nullptr, nullptr, g, scale))) return rc;
    // (also writes dD1, the restriction of dS0)
    if ((rc = conv_dgrad(net, DEC0, nullptr, g, net->dS0))) return rc;
    if ((rc = conv_wgrad(net, DEC1, net->S1, nullptr, net->dD1, nullptr, scale))) return rc;
    if ((rc = conv_dgrad(net, DEC1, net->dD1, nullptr, net->dS1))) return rc;
    if ((rc = restrict_to<32>(net, 1, net->dS1, net->dD2, 1.f))) return rc;
    if ((rc = conv_wgrad(net, DEC2, net->S2, nullptr, net->dD2, nullptr, scale))) return rc;
    if ((rc = conv_dgrad(net, DEC2, net->dD2, nullptr, net->dS2))) return rc;
    if ((rc = restrict_to<64>(net, 2, net->dS2, net->dD3, 1.f))) return rc;
    if ((rc = conv_wgrad(net, DEC3, net->E3, nullptr, net->dD3, nullptr, scale))) return rc;
    if ((rc = conv_dgrad(net, DEC3, net->dD3, nullptr, net->dE3))) return rc;
    if ((rc = conv_wgrad(net, ENC3, net->P3, nullptr, net->dE3, nullptr, scale))) return rc;
    if ((rc = conv_dgrad(net, ENC3, net->dE3, nullptr, net->dP3))) return rc;
    if ((rc = prolong_add<64>(net, 2, net->dP3, net->dS2, 0.125f))) return rc;
    if ((rc = conv_wgrad(net, ENC2, net->P2, nullptr, net->dS2, nullptr, scale))) return rc;
    if ((rc = conv_dgrad(net, ENC2, net->dS2, nullptr, net->dP2))) return rc;
    if ((rc = prolong_add<32>(net, 1, net->dP2, net->dS1, 0.125f))) return rc;
    if ((rc = conv_wgrad(net, ENC1, net->P1, nullptr, net->dS1, nullptr, scale))) return rc;
    if ((rc = conv_dgrad(net, ENC1, net->dS1, nullptr, net->dP1))) return rc;
    if ((rc = prolong_add<16>(net, 0, net->dP1, net->dS0, 0.125f))) return rc;
    return conv_wgrad(net, ENC0, nullptr, u, net->dS0, nullptr, scale);
}

static int pack_weights(dare_unet* net) {
    dare_ctx* ctx = net->ctx;
    k_pack_tapk<<<1, 256, 0, ctx->stream>>>(net->w + net->layer[ENC0].woff, 0, net->layer[ENC0].wf);
    DARE_LAUNCHED(ctx);
    k_pack_tapn<<<1, 256, 0, ctx->stream>>>(net->w + net->layer[DEC0].woff, net->layer[DEC0].wf);
    DARE_LAUNCHED(ctx);
    k_pack_tapk<<<1, 256, 0, ctx->stream>>>(net->w + net->layer[DEC0].woff, 1, net->layer[DEC0].wb);
    DARE_LAUNCHED(ctx);
    for (int l = ENC1; l <= DEC1; l++) {
        Layer& L = net->layer[l];
        const int nz = L.coutk / L.nt;
        k_pack<<<eblocks(ctx, (int64_t)nz * kTaps * L.cink * L.nt), 256, 0, ctx->stream>>>(
            net->w + L.woff, L.cin, L.cout, L.cink, L.nt, nz, 0, L.wf);
        DARE_LAUNCHED(ctx);
        if (l != ENC0) {
            const int nzb = L.cink / L.ntb;
            k_pack<<<eblocks(ctx, (int64_t)nzb * kTaps * L.coutk * L.ntb), 256, 0, ctx->stream>>>(
                net->w + L.woff, L.cin, L.cout, L.coutk, L.ntb, nzb, 1, L.wb);
            DARE_LAUNCHED(ctx);
        }
    }
    return DARE_OK;
}

// Reads the device error word of the launches so far; a reported time-out is
// cleared, so the network stays usable for the next call.
static int check_err(dare_unet* net) {
    int e = 0;
    DARE_CUDA(net->ctx, cudaMemcpyAsync(&e, net->err, sizeof(int), cudaMemcpyDeviceToHost, net->ctx->stream));
    DARE_CUDA(net->ctx, cudaStreamSynchronize(net->ctx->stream));
    if (e) {
        DARE_CUDA(net->ctx, cudaMemsetAsync(net->err, 0, sizeof(int), net->ctx->stream));
        return set_error(net->ctx, DARE_ERR_TIMEOUT,
                         "unet: a tensor-core wait timed out (code " + std::to_string(e) + ")");
    }
    return DARE_OK;
}

// Mean loss and gradient over `count` pairs; grad is zeroed first.
static int loss_grad(dare_unet* net, const float* const* r, const float* const* e, const float* const* en2, int count,
                     double* loss) {
    dare_ctx* ctx = net->ctx;
    int rc;
    DARE_CUDA(ctx, cudaMemsetAsync(net->grad, 0, net->nparam * sizeof(float), ctx->stream));
    DARE_CUDA(ctx, cudaMemsetAsync(net->dscal, 0, sizeof(double), ctx->stream));
    const float scale = 1.f / (float)count;
    for (int b = 0; b < count; b++) {
        if ((rc = apply_grid(net, r[b], net->z))) return rc;   // pairs live on the network's grid
        k_loss_grad<<<eblocks(ctx, net->ncell), 256, 0, ctx->stream>>>(net->ncell, net->z, e[b], en2[b], scale,
                                                                       net->g, net->dscal);
        DARE_LAUNCHED(ctx);
        if ((rc = backward(net, r[b], net->g, 1.f))) return rc;
    }
    if (loss) {
        DARE_CUDA(ctx, cudaMemcpyAsync(loss, net->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    return check_err(net);
}

static int adam_step(dare_unet* net, const dare_unet_train_params* p) {
    dare_ctx* ctx = net->ctx;
    net->adam_t++;
    const float bc1 = 1.f - powf(p->beta1, (float)net->adam_t);
    const float bc2 = 1.f - powf(p->beta2, (float)net->adam_t);
    k_adam<<<eblocks(ctx, net->nparam), 256, 0, ctx->stream>>>(net->nparam, net->w, net->grad, net->adam_m,
                                                               net->adam_v, p->lr, p->beta1, p->beta2, p->eps, bc1, bc2);
    DARE_LAUNCHED(ctx);
    net->steps++;
    return pack_weights(net);
}

// ||e||^2 of device pairs into out[b] (for the public loss calls)
static int pair_norms(dare_unet* net, const float* e, int count, float* out) {
    dare_ctx* ctx = net->ctx;
    for (int b = 0; b < count; b++) {
        DARE_CUDA(ctx, cudaMemsetAsync(net->dscal + 1, 0, sizeof(double), ctx->stream));
        k_sqnorm<<<eblocks(ctx, net->ncell), 256, 0, ctx->stream>>>(net->ncell, e + (size_t)b * net->ncell,
                                                                    net->dscal + 1);
        DARE_LAUNCHED(ctx);
        k_store_norm<<<1, 1, 0, ctx->stream>>>(net->dscal + 1, out + b);
        DARE_LAUNCHED(ctx);
    }
    return DARE_OK;
}

}  // namespace unet
}  // namespace dare_gpu

// ===========================================================================
// C ABI
extern "C" {

void dare_unet_train_params_default(dare_unet_train_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->lr = 2e-4f;
    p->beta1 = 0.9f;
    p->beta2 = 0.999f;
    p->eps = 1e-8f;
    p->batch = 4;
    p->steps = 8;
    p->max_pairs_per_rhs = 12;
    p->seed = 1234;
}

static void unet_free(dare_unet* net) {
    for (int l = 0; l < kLayers; l++) {
        cudaFree(net->layer[l].wf);
        cudaFree(net->layer[l].wb);
    }
    cudaFree(net->w);
    cudaFree(net->grad);
    cudaFree(net->adam_m);
    cudaFree(net->adam_v);
    cudaFree(net->act_block);
    cudaFree(net->X0);
    cudaFree(net->z);
    cudaFree(net->g);
    cudaFree(net->part);
    cudaFree(net->dscal);
    cudaFree(net->err);
    cudaFree(net->ring_r);
    cudaFree(net->ring_e);
    cudaFree(net->ring_en);
    cudaFree(net->sol);
    cudaFree(net->cbuf);
    cudaFree(net->fbuf);
}

int dare_unet_create(dare_ctx* ctx, const int n[3], uint64_t seed, dare_unet** out) {
    if (!ctx || !n || !out) return DARE_ERR_BAD_ARG;
    *out = nullptr;
    for (int d = 0; d < 3; d++)
        if (n[d] < 8 || n[d] % 8 != 0)
            return set_error(ctx, DARE_ERR_BAD_ARG, "dare_unet_create: every grid size must be a positive multiple of 8");
    if (n[2] + 2 + 8 >= kActSlackRows)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "dare_unet_create: grid too wide for the staged convolutions");
    cudaSetDevice(ctx->device);
    dare_unet* net = new dare_unet();
    net->ctx = ctx;
    net->device = ctx->device;
    for (int d = 0; d < 3; d++) net->n[d] = n[d];
    net->ncell = (int64_t)n[0] * n[1] * n[2];
    for (int l = 0; l < kLevels; l++) net->geo[l] = make_geom(n[0] >> l, n[1] >> l, n[2] >> l);
    int64_t off = 0;
    for (int l = 0; l < kLayers; l++) {
        Layer& L = net->layer[l];
        L.level = kDefs[l].level;
        L.cin = kDefs[l].cin;
        L.cout = kDefs[l].cout;
        L.cink = std::max(L.cin, 16);
        L.coutk = std::max(L.cout, 16);
        const Geom& g = net->geo[L.level];
        L.nt = pick_nt(L.cink, L.coutk, g);
        L.ntb = pick_nt(L.coutk, L.cink, g);
        const bool fits_fwd = l == ENC0   ? in_smem(kInMT) <= kMaxSmem
                              : l == DEC0 ? out_smem(g, 1, 2) <= kMaxSmem
                                          : fwd_smem(L.cink, L.nt, g, 1, 4) <= kMaxSmem;
        const bool fits_bwd = l == ENC0   ? true
                              : l == DEC0 ? in_smem(kInMT) <= kMaxSmem
                                          : fwd_smem(L.coutk, L.ntb, g, 1, 4) <= kMaxSmem;
        if (!fits_fwd || !fits_bwd || wgr_smem(L.cink, L.coutk, g, l == ENC0, l == DEC0) > kMaxSmem) {
            delete net;
            return set_error(ctx, DARE_ERR_UNSUPPORTED, "dare_unet_create: grid too wide for the staged convolutions");
        }
        L.woff = off;
        L.nparam = (int64_t)kTaps * L.cin * L.cout;
        off += L.nparam;
    }
    net->nparam = off;

    // activations: one zeroed block, every buffer 256-byte aligned
    const int64_t T[4] = {net->geo[0].total, net->geo[1].total, net->geo[2].total, net->geo[3].total};
    struct Slot {
        bf16** p;
        int level, c, extra;
    } slots[] = {{&net->S0, 0, 16}, {&net->P1, 1, 16}, {&net->S1, 1, 32}, {&net->P2, 2, 32}, {&net->S2, 2, 64},
                 {&net->P3, 3, 64}, {&net->E3, 3, 64}, {&net->dS0, 0, 16}, {&net->dD1, 1, 16}, {&net->dS1, 1, 32},
                 {&net->dD2, 2, 32}, {&net->dS2, 2, 64}, {&net->dD3, 3, 64}, {&net->dE3, 3, 64}, {&net->dP3, 3, 64},
                 {&net->dP2, 2, 32}, {&net->dP1, 1, 16}};
    // a staged plane segment reaches up to W + 8 rows before the start of an
    // array (the unused halo of the ghost plane 0) and kActSlackRows bounds W
    size_t bytes = (size_t)kActSlackRows * 16;
    std::vector<size_t> offs;
    for (auto& s : slots) {
        offs.push_back(bytes);
        bytes += (((size_t)T[s.level] * s.c + s.extra) * sizeof(bf16) + 255) / 256 * 256;
    }
    bytes += (size_t)kActSlackRows * 16;  // rows a staged segment may read past the last array
    cudaError_t e = cudaMalloc(&net->act_block, bytes);
    if (e == cudaSuccess) e = cudaMemset(net->act_block, 0, bytes);
    for (size_t i = 0; i < sizeof(slots) / sizeof(slots[0]) && e == cudaSuccess; i++)
        *slots[i].p = reinterpret_cast<bf16*>(static_cast<uint8_t*>(net->act_block) + offs[i]);
    const size_t pb = net->nparam * sizeof(float);
    // (grid sizes are multiples of 8, so the pitched copy is only for a
    // caller's vector that does not start on a 16-byte boundary)
    if (e == cudaSuccess) e = cudaMalloc(&net->X0, (size_t)net->ncell * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&net->w, pb);
    if (e == cudaSuccess) e = cudaMalloc(&net->grad, pb);
    if (e == cudaSuccess) e = cudaMalloc(&net->adam_m, pb);
    if (e == cudaSuccess) e = cudaMalloc(&net->adam_v, pb);
    if (e == cudaSuccess) e = cudaMemset(net->adam_m, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(net->adam_v, 0, pb);
    if (e == cudaSuccess) e = cudaMalloc(&net->z, net->ncell * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(net->z, 0, net->ncell * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&net->g, net->ncell * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&net->dscal, 4 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&net->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(net->err, 0, sizeof(int));
    for (int l = 0; l < kLayers && e == cudaSuccess; l++) {
        Layer& L = net->layer[l];
        e = cudaMalloc(&L.wf, (size_t)kTaps * L.cink * L.coutk * sizeof(bf16));
        if (e == cudaSuccess && l != ENC0) e = cudaMalloc(&L.wb, (size_t)kTaps * L.cink * L.coutk * sizeof(bf16));
    }
    if (e != cudaSuccess) {
        unet_free(net);
        delete net;
        return check_cuda(ctx, e, "dare_unet_create");
    }
    // initial weights: N(0, 1/(27 cin)) per layer (variance-preserving for a
    // linear network); dec0 zero so that N = I before training
    std::vector<float> h(net->nparam, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < kLayers; l++) {
        const Layer& L = net->layer[l];
        if (l == DEC0) continue;
        std::normal_distribution<float> nd(0.f, 1.f / std::sqrt((float)(kTaps * L.cin)));
        for (int64_t i = 0; i < L.nparam; i++) h[L.woff + i] = nd(rng);
    }
    net->rng = seed * 0x9E3779B97F4A7C15ull + 1;
    int rc = dare_unet_set_weights(net, h.data(), net->nparam);
    if (rc) {
        unet_free(net);
        delete net;
        return rc;
    }
    *out = net;
    return DARE_OK;
}

int dare_unet_create_coarse(dare_ctx* ctx, const int n_fine[3], uint64_t seed, dare_unet** out) {
    if (!ctx || !n_fine || !out) return DARE_ERR_BAD_ARG;
    *out = nullptr;
    int nc[3];
    for (int d = 0; d < 3; d++) {
        if (n_fine[d] < 16 || n_fine[d] % 16 != 0)
            return set_error(ctx, DARE_ERR_BAD_ARG,
                             "dare_unet_create_coarse: every grid size must be a positive multiple of 16");
        nc[d] = n_fine[d] / 2;
    }
    dare_unet* net = nullptr;
    int rc = dare_unet_create(ctx, nc, seed, &net);
    if (rc) return rc;
    net->coarse = 1;
    for (int d = 0; d < 3; d++) net->fine[d] = n_fine[d];
    net->fine_ncell = (int64_t)n_fine[0] * n_fine[1] * n_fine[2];
    cudaError_t e = cudaMalloc(&net->cbuf, (size_t)net->ncell * 2 * sizeof(float));
    if (e != cudaSuccess) {
        dare_unet_destroy(net);
        return check_cuda(ctx, e, "dare_unet_create_coarse");
    }
    *out = net;
    return DARE_OK;
}

int dare_unet_system_shape(const dare_unet* net, int n[3]) {
    if (!net || !n) return DARE_ERR_BAD_ARG;
    for (int d = 0; d < 3; d++) n[d] = net->coarse ? net->fine[d] : net->n[d];
    return net->coarse;
}

int dare_unet_set_wait_limit(dare_unet* net, int64_t polls) {
    if (!net || polls < 0 || polls > 0xFFFFFFFFll) return DARE_ERR_BAD_ARG;
    net->wait_limit = polls == 0 ? kWaitLimit : (uint32_t)polls;
    return DARE_OK;
}

int dare_unet_debug_skip_plane(dare_unet* net) {
    if (!net) return DARE_ERR_BAD_ARG;
    net->debug_skip = 1;
    return DARE_OK;
}

int dare_unet_destroy(dare_unet* net) {
    if (!net) return DARE_OK;
    cudaSetDevice(net->device);
    unet_free(net);
    delete net;
    return DARE_OK;
}

int64_t dare_unet_num_params(const dare_unet* net) { return net ? net->nparam : 0; }

int dare_unet_get_weights(dare_unet* net, float* host, int64_t count) {
    if (!net || !host || count != net->nparam) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = net->ctx;
    cudaSetDevice(ctx->device);
    DARE_CUDA(ctx, cudaMemcpyAsync(host, net->w, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_unet_set_weights(dare_unet* net, const float* host, int64_t count) {
    if (!net || !host || count != net->nparam) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = net->ctx;
    cudaSetDevice(ctx->device);
    DARE_CUDA(ctx, cudaMemcpyAsync(net->w, host, count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    int rc = pack_weights(net);
    if (rc) return rc;
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_unet_apply(dare_unet* net, const float* u, float* z) {
    if (!net || !u || !z || u == z) return DARE_ERR_BAD_ARG;
    cudaSetDevice(net->ctx->device);
    int rc = apply(net, u, z);
    if (rc) return rc;
    return check_err(net);
}

int dare_unet_read_activation(dare_unet* net, int which, float* host, int64_t count) {
    if (!net || !host || which < 0 || which > 6) return DARE_ERR_BAD_ARG;
    static const int lev[7] = {0, 1, 1, 2, 2, 3, 3}, ch[7] = {16, 16, 32, 32, 64, 64, 64};
    bf16* const buf[7] = {net->S0, net->P1, net->S1, net->P2, net->S2, net->P3, net->E3};
    const Geom& g = net->geo[lev[which]];
    const int64_t total = (int64_t)g.n0 * g.n1 * g.n2 * ch[which];
    if (count != total) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = net->ctx;
    cudaSetDevice(ctx->device);
    float* d = nullptr;
    DARE_CUDA(ctx, cudaMalloc(&d, total * sizeof(float)));
    k_read_act<<<eblocks(ctx, total), 256, 0, ctx->stream>>>(g, ch[which], buf[which], d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, total * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return check_cuda(ctx, e, "dare_unet_read_activation");
    return DARE_OK;
}

int dare_unet_loss_grad(dare_unet* net, const float* r, const float* e, int count, double* loss, float* grad_host) {
    if (!net || !r || !e || count < 1) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = net->ctx;
    cudaSetDevice(ctx->device);
    float* en2 = nullptr;
    DARE_CUDA(ctx, cudaMalloc(&en2, count * sizeof(float)));
    int rc = pair_norms(net, e, count, en2);
    std::vector<const float*> rp(count), ep(count), np(count);
    for (int b = 0; b < count; b++) {
        rp[b] = r + (size_t)b * net->ncell;
        ep[b] = e + (size_t)b * net->ncell;
        np[b] = en2 + b;
    }
    double l = 0.;
    if (!rc) rc = loss_grad(net, rp.data(), ep.data(), np.data(), count, &l);
    if (!rc && grad_host) {
        cudaError_t ce = cudaMemcpyAsync(grad_host, net->grad, net->nparam * sizeof(float), cudaMemcpyDeviceToHost,
                                         ctx->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
        if (ce != cudaSuccess) rc = check_cuda(ctx, ce, "dare_unet_loss_grad");
    }
    cudaFree(en2);
    if (loss) *loss = l;
    return rc;
}

int dare_unet_train_step(dare_unet* net, const float* r, const float* e, int count, const dare_unet_train_params* p,
                         double* loss) {
    if (!net || !r || !e || !p || count < 1) return DARE_ERR_BAD_ARG;
    int rc = dare_unet_loss_grad(net, r, e, count, loss, nullptr);
    if (rc) return rc;
    if ((rc = adam_step(net, p))) return rc;
    DARE_CUDA(net->ctx, cudaStreamSynchronize(net->ctx->stream));
    return DARE_OK;
}

int dare_unet_launch_info(const dare_unet* net, int layer, int kind, int64_t info[8]) {
    if (!net || !info || layer < 0 || layer >= kLayers || kind < 0 || kind > 2) return DARE_ERR_BAD_ARG;
    const Layer& L = net->layer[layer];
    const LaunchCfg& c = kind == 0 ? L.fwd : (kind == 1 ? L.bwd : L.wgr);
    if (!c.ready) return DARE_ERR_STATE;
    const int64_t v[8] = {c.grid.x, c.grid.y, c.grid.z, (int64_t)c.smem, c.ppc, kind == 2 ? c.tpg : c.slots, c.cols,
                          c.occ};
    for (int i = 0; i < 8; i++) info[i] = v[i];
    return DARE_OK;
}

int dare_unet_stats(const dare_unet* net, int64_t* steps, int64_t* pairs_seen) {
    if (!net) return DARE_ERR_BAD_ARG;
    if (steps) *steps = net->steps;
    if (pairs_seen) *pairs_seen = net->pairs_seen;
    return DARE_OK;
}

int dare_unet_train_on_system(dare_unet* net, dare_system* s, double tol, const dare_unet_train_params* p,
                              dare_unet_train_report* rep) {
    if (!net || !s || !p || !rep || p->batch < 1 || p->steps < 0) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = net->ctx;
    const GridDev& g = s->grid->dev;
    const int* sys_n = net->coarse ? net->fine : net->n;
    if (g.dim != 3 || g.n[0] != sys_n[0] || g.n[1] != sys_n[1] || g.n[2] != sys_n[2])
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_unet_train_on_system: grid does not match the network");
    if (s->ncomp != 1)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "dare_unet_train_on_system: one field component only");
    cudaSetDevice(ctx->device);
    std::memset(rep, 0, sizeof(*rep));
    const int64_t n = net->ncell;                           // pairs in the ring: the network's grid
    const int64_t nf = net->coarse ? net->fine_ncell : n;   // the system's grid
    if (!net->ring_r) {
        // ring of pairs: up to 256 (2048 for the coarse form), at most ~4 GB
        const size_t pair_bytes = (size_t)n * 2 * sizeof(float);
        const size_t most = net->coarse ? 2048 : 256;
        int cap = (int)std::min<size_t>(most, std::max<size_t>(8, ((size_t)4 << 30) / pair_bytes));
        cudaError_t e = cudaMalloc(&net->ring_r, (size_t)cap * n * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&net->ring_e, (size_t)cap * n * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&net->ring_en, (size_t)cap * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&net->sol, (size_t)2 * nf * sizeof(double));
        if (e == cudaSuccess && net->coarse) e = cudaMalloc(&net->fbuf, (size_t)2 * nf * sizeof(float));
        if (e != cudaSuccess) return check_cuda(ctx, e, "dare_unet_train_on_system");
        net->ring_cap = cap;
    }
    double* x0 = net->sol;
    double* xs = net->sol + nf;
    const int eb = eblocks(ctx, nf);
    DARE_CUDA(ctx, cudaMemcpyAsync(x0, s->x, nf * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));

    // the plain solve to the tolerance, warm-started at x0
    dare_solver_params sp;
    dare_solver_params_default(&sp);
    sp.tol = tol;
    sp.tol_relative = 1;
    sp.max_it = 1000;
    sp.compute_true_residual = 0;
    dare_solve_report sr;
    k_warm<<<eb, 256, 0, ctx->stream>>>(nf, s->diag, x0, s->x);
    DARE_LAUNCHED(ctx);
    int rc = dare_bicgstab2_fp64(s, &sp, &sr);
    if (rc) return rc;
    rep->plain_iters = sr.iters;
    DARE_CUDA(ctx, cudaMemcpyAsync(xs, s->x, nf * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));

    // its iterates x_k, k = 0 .. K-1, as pairs; the coarse form keeps their
    // restrictions (the fine loss ||r + P U(R r) - e||^2 is 8 ||R r + U(R r)
    // - R e||^2 plus a term without U, for the average R and the nearest P)
    const int K = std::min(std::max(sr.iters, 1), p->max_pairs_per_rhs);
    for (int k = 0; k < K; k++) {
        const double* xk = x0;
        if (k > 0) {
            dare_solver_params q = sp;
            q.tol = 0.;
            q.tol_relative = 0;
            q.max_it = k;
            k_warm<<<eb, 256, 0, ctx->stream>>>(nf, s->diag, x0, s->x);
            DARE_LAUNCHED(ctx);
            dare_solve_report qr;
            if ((rc = dare_bicgstab2_fp64(s, &q, &qr))) return rc;
            xk = s->x;
        }
        const int slot = net->ring_next;
        float* rs = net->ring_r + (size_t)slot * n;
        float* es = net->ring_e + (size_t)slot * n;
        DARE_CUDA(ctx, cudaMemsetAsync(net->dscal + 2, 0, sizeof(double), ctx->stream));
        k_make_pair<<<eb, 256, 0, ctx->stream>>>(g, s->diag, s->rhs, xk, xs, net->coarse ? net->fbuf : rs,
                                                 net->coarse ? net->fbuf + nf : es, net->dscal + 2);
        DARE_LAUNCHED(ctx);
        if (net->coarse) {
            k_pool8<<<eblocks(ctx, n / 2), 256, 0, ctx->stream>>>(net->n[0], net->n[1], net->n[2], net->fbuf, rs);
            DARE_LAUNCHED(ctx);
            k_pool8<<<eblocks(ctx, n / 2), 256, 0, ctx->stream>>>(net->n[0], net->n[1], net->n[2], net->fbuf + nf, es);
            DARE_LAUNCHED(ctx);
            DARE_CUDA(ctx, cudaMemsetAsync(net->dscal + 2, 0, sizeof(double), ctx->stream));
            k_sqnorm<<<eblocks(ctx, n), 256, 0, ctx->stream>>>(n, es, net->dscal + 2);
            DARE_LAUNCHED(ctx);
        }
        k_store_norm<<<1, 1, 0, ctx->stream>>>(net->dscal + 2, net->ring_en + slot);
        DARE_LAUNCHED(ctx);
        net->ring_next = (net->ring_next + 1) % net->ring_cap;
        net->ring_size = std::min(net->ring_size + 1, net->ring_cap);
        rep->pairs_added++;
        net->pairs_seen++;
    }
    DARE_CUDA(ctx, cudaMemcpyAsync(s->x, xs, nf * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));

    // optimiser steps on minibatches drawn from the ring
    std::mt19937_64 rng(p->seed ^ net->rng);
    net->rng = net->rng * 6364136223846793005ull + 1442695040888963407ull;
    std::vector<const float*> rp(p->batch), ep(p->batch), np(p->batch);
    for (int st = 0; st < p->steps; st++) {
        for (int b = 0; b < p->batch; b++) {
            const int i = (int)(rng() % (uint64_t)net->ring_size);
            rp[b] = net->ring_r + (size_t)i * n;
            ep[b] = net->ring_e + (size_t)i * n;
            np[b] = net->ring_en + i;
        }
        double l = 0.;
        if ((rc = loss_grad(net, rp.data(), ep.data(), np.data(), p->batch, &l))) return rc;
        if (st == 0) rep->loss_first = l;
        rep->loss_last = l;
        if ((rc = adam_step(net, p))) return rc;
        rep->steps++;
    }
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    rep->pairs_total = net->ring_size;
    return DARE_OK;
}

}  // extern "C"
