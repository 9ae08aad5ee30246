// dare_noalloc.cu -- the residual norm ||b - A x||_2 of a structured 7-point
// system without any device allocation.
//
// Who needs it: a host code that embeds this solver inside its own time loop
// often owns all device memory through its own allocator or fixed budget,
// and cannot afford cudaMalloc there: cudaMalloc synchronizes the device
// (stalling every other stream of the application) and may fail at an
// arbitrary step when memory is tight.  This entry point takes the operator
// and vectors as plain device pointers, writes the norm to a device pointer,
// and keeps its only scratch -- the per-item partial sums and the work-queue
// counters of the marching kernel -- in a fixed file-scope device array.
//
// Limits and sharing rules:
//   * the scratch holds kNoAllocMaxItems partial sums; grids whose (j,k)
//     plane needs more tiles than that (ny*nz above ~1M cells) are rejected;
//   * every call on a device uses the same array and it keeps the last
//     call's contents; the counters are cleared at the start of each call on
//     the caller's stream.  Calls that overlap on the GPU (different streams,
//     or host threads) race on the array and must be serialized by the caller;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current), so make that first
//     call before any stream capture is started on the device.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "dare_march.cuh"

using namespace dare_gpu;

namespace {

constexpr int kNoAllocMaxItems = 4096;
constexpr size_t kStateBytes = 256;  // SolverState, padded
constexpr size_t kScratchBytes = kStateBytes + sizeof(double) * kNoAllocMaxItems;
static_assert(sizeof(SolverState) <= kStateBytes, "state slot too small");

// The scratch: counters first, then the partial sums.  Host code must never
// use the symbol itself as an address (it names a host-side stand-in); the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_dev[kMaxDevices] = {nullptr};
int g_num_sms[kMaxDevices] = {0};

int fail(char* err, int err_len, int code, const char* msg) {
    if (err && err_len > 0) {
        std::strncpy(err, msg, (size_t)err_len - 1);
        err[err_len - 1] = '\0';
    }
    return code;
}

}  // namespace

extern "C" int dare_residual_norm_noalloc(int dim, const int64_t n[3], const int periodic[3], const double* diag7,
                                          const double* x, const double* b, double* norm_out, void* stream,
                                          char* err, int err_len) {
    if (err && err_len > 0) err[0] = '\0';
    if (dim < 1 || dim > 3 || !n || !diag7 || !x || !b || !norm_out)
        return fail(err, err_len, DARE_ERR_BAD_ARG, "dare_residual_norm_noalloc: bad arguments");
    GridDev g{};
    g.dim = dim;
    int64_t total = 1;
    for (int d = 0; d < 3; d++) {
        const int64_t nd = d < dim ? n[d] : 1;
        if (nd < 1 || nd > (1 << 30)) return fail(err, err_len, DARE_ERR_BAD_ARG, "dare_residual_norm_noalloc: bad size");
        g.n[d] = (int)nd;
        g.gn[d] = (int)nd;
        g.periodic[d] = (d < dim && periodic) ? (periodic[d] != 0) : 0;
        total *= nd;
    }
    if (total >= ((int64_t)1 << 31)) return fail(err, err_len, DARE_ERR_UNSUPPORTED, "dare_residual_norm_noalloc: more than 2^31 cells");
    g.ncell = total;
    g.ncell_ghosted = total;

    // work items: 32x8 (j,k) tiles (narrower for thin grids) and plane runs,
    // at most kNoAllocMaxItems of them
    MarchCfg m;
    const int tk = g.n[2] > 16 ? 32 : g.n[2] > 8 ? 16 : g.n[2] > 4 ? 8 : g.n[2] > 2 ? 4 : 1;
    int tj = 256 / tk;
    while (tj > 1 && tj / 2 >= g.n[1]) tj /= 2;
    m.block = dim3(tk, tj, 1);
    m.tiles_x = (g.n[2] + tk - 1) / tk;
    m.tiles_y = (g.n[1] + tj - 1) / tj;
    const int64_t tiles = (int64_t)m.tiles_x * m.tiles_y;
    if (tiles > kNoAllocMaxItems)
        return fail(err, err_len, DARE_ERR_UNSUPPORTED,
                    "dare_residual_norm_noalloc: the (j,k) plane needs more than 4096 tiles of 32x8 cells "
                    "(ny*nz above about 1M); use the allocating solver path");
    int planes = 32;
    while (tiles * ((g.n[0] + planes - 1) / planes) > kNoAllocMaxItems) planes *= 2;
    if (planes > g.n[0]) planes = g.n[0];
    m.planes = planes;
    m.nitems = (int)(tiles * ((g.n[0] + planes - 1) / planes));

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return fail(err, err_len, DARE_ERR_CUDA, "dare_residual_norm_noalloc: no current device");
    }
    void* scratch = nullptr;
    int num_sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch_dev[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return fail(err, err_len, DARE_ERR_CUDA, "dare_residual_norm_noalloc: cudaGetSymbolAddress failed");
            }
            int sms = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
            g_num_sms[dev] = sms;
            g_scratch_dev[dev] = p;
        }
        scratch = g_scratch_dev[dev];
        num_sms = g_num_sms[dev];
    }
    SolverState* st = reinterpret_cast<SolverState*>(scratch);
    double* partials = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + kStateBytes);
    cudaStream_t sm = (cudaStream_t)stream;

    // the reduction and queue counters must start at zero
    if (cudaMemsetAsync(st, 0, sizeof(SolverState), sm) != cudaSuccess) {
        cudaGetLastError();
        return fail(err, err_len, DARE_ERR_CUDA, "dare_residual_norm_noalloc: clearing the counters failed");
    }
    const int64_t nc = g.ncell;
    OpT<double> op{diag7, diag7 + nc, nc};
    FResidual<double> f{};
    f.zs[0] = x;
    set_coef_streams<double, false, 8>(op, f.ps);
    f.ps[7] = b;
    f.out = norm_out;
    const size_t smem = march_smem_bytes<FResidual<double>>(m);
    int per_sm = 0;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_march<FResidual<double>>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess) {
        cudaGetLastError();
        return fail(err, err_len, DARE_ERR_CUDA, "dare_residual_norm_noalloc: shared memory attribute");
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_march<FResidual<double>>, m.block.x * m.block.y, smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * num_sms;
    if (blocks > m.nitems) blocks = m.nitems;
    k_march<FResidual<double>><<<blocks, m.block, smem, sm>>>(g, f, st, partials, m);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(err, err_len, DARE_ERR_CUDA, cudaGetErrorString(e));
    return DARE_OK;
}
