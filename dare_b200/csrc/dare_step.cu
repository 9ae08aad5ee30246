// dare_step.cu -- one implicit time step of the reference's driver loop
// (test/Verification/counter_diffusion1D.cpp:170-217 and
// advection_periodic2D.cpp:160-196): Build, Solve, CopyTo,
// ExchangeHaloCells, CopyDataVectorsToOldTimeStep -- all on the device,
// control returning to the host only for the solver's status.
#include <cstring>

#include "dare_internal.cuh"

using namespace dare_gpu;

extern "C" int dare_bicgstab2_solve_to_field(dare_system* s, const dare_solver_params* p, dare_solve_report* rep,
                                             dare_field* f, int* field_written);
namespace dare_gpu {
int launch_assemble(dare_system* s, const dare_assembly_desc* desc, const double* phi, const double* phi_old);
int launch_assemble_planes(dare_system* s, const dare_assembly_desc* desc, const double* phi, const double* phi_old,
                           int ib, int ie);
int launch_scatter(dare_ctx* ctx, const GridDev& g, const double* x, double* phi);
int launch_halo(dare_ctx* ctx, const GridDev& g, double* phi);
}  // namespace dare_gpu

extern "C" {

int dare_timestep(dare_system* s, dare_field* f, const dare_assembly_desc* desc, const dare_solver_params* p,
                  dare_solve_report* rep) {
    if (!s || !f || !desc || !p || !rep || f->grid != s->grid || f->ncomp != s->ncomp) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = s->grid->ctx;
    cudaSetDevice(ctx->device);
    const double* phi = f->level[0];
    const double* phi_old = f->num_levels > 1 ? f->level[1] : f->level[0];
    const bool prof = ctx->profiling != 0;
    if (prof) DARE_CUDA(ctx, cudaEventRecord(ctx->ev[12], ctx->stream));
    int rc = launch_assemble(s, desc, phi, phi_old);                 // Trilinos::Build
    if (rc) return rc;
    if (prof) DARE_CUDA(ctx, cudaEventRecord(ctx->ev[13], ctx->stream));
    int written = 0;                                                 // TrilinosSolver::Solve, and with the
    rc = dare_bicgstab2_solve_to_field(s, p, rep, f, &written);      // plain FP64 solve CopyTo and
    if (rc) return rc;                                               // ExchangeHaloCells at its exit
    if (prof) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev[12], ctx->ev[13]) == cudaSuccess) {
            ctx->stat_ms[KID_ASSEMBLE] += ms;
            ctx->stat_n[KID_ASSEMBLE] += 1;
        } else {
            cudaGetLastError();
        }
    }
    if (!written) {
        rc = dare_system_copy_to(s, f);                               // Trilinos::CopyTo
        if (rc) return rc;
        rc = dare_field_exchange_halo(f);                             // Field::ExchangeHaloCells
        if (rc) return rc;
    }
    return dare_field_copy_to_old(f);                                // CopyDataVectorsToOldTimeStep
}

}  // extern "C"

namespace {
// The rest of a step whose Build has been queued: Solve, CopyTo,
// ExchangeHaloCells (CopyDataVectorsToOldTimeStep is the caller's).
int solve_and_copy_back(dare_system* s, dare_field* f, const dare_solver_params* p, dare_solve_report* rep) {
    int written = 0;
    int rc = dare_bicgstab2_solve_to_field(s, p, rep, f, &written);
    if (rc || written) return rc;
    rc = dare_system_copy_to(s, f);
    if (rc) return rc;
    return dare_field_exchange_halo(f);
}
}  // namespace

extern "C" {

// nsteps steps of a field that lives in host memory: before step k the
// field's level 0 is read from `host` and level 1 set from it; after the step
// the result goes back to `host`.  The host buffer is in the field's device
// layout (component-major ghosted levels) and must be pinned.  The result of
// step k travels to the host and the input of step k + 1 back to the device
// in kHostChunks slices on two streams: slice c goes up as soon as it has
// come down, so the two PCIe directions run at the same time instead of one
// after the other.  Every step still moves the whole field both ways.  On
// single-component 3-D grids the step's Build runs under the upload: each
// slice, once on the device, is copied to level 1 and the planes whose
// stencil it completes are assembled (256^3: 66.9 -> 69.1 steps/s end to
// end); the fields and coefficients are those of the loop of single calls,
// bit for bit.
int dare_timesteps_host(dare_system* s, dare_field* f, const dare_assembly_desc* desc, const dare_solver_params* p,
                        int nsteps, double* host, dare_solve_report* reps) {
    if (!s || !f || !desc || !p || !host || nsteps < 1 || f->grid != s->grid || f->ncomp != s->ncomp)
        return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = s->grid->ctx;
    cudaSetDevice(ctx->device);
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, host) != cudaSuccess || attr.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_timesteps_host: the host buffer must be pinned");
    }
    constexpr int kHostChunks = 16;
    const GridDev& gd = f->grid->dev;
    const size_t total = (size_t)gd.ncell_ghosted * f->ncomp * sizeof(double);
    size_t chunk = (total + kHostChunks - 1) / kHostChunks;
    chunk = (chunk + 4095) / 4096 * 4096;
    char* dev = reinterpret_cast<char*>(f->level[0]);
    char* hb = reinterpret_cast<char*>(host);
    // Single-component 3-D grids with an old level: each slice, once on the
    // device, is copied to the old level and the planes whose stencil it
    // completes are assembled at once, so the assembly runs under the rest of
    // the upload (the coefficients of every plane are those of one launch).
    const bool sliced = gd.dim == 3 && f->ncomp == 1 && f->num_levels > 1 && s->ncomp == 1;
    char* dev_old = sliced ? reinterpret_cast<char*>(f->level[1]) : nullptr;
    const size_t plane_bytes = (size_t)gd.gn[1] * gd.gn[2] * sizeof(double);
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t ev_in = nullptr, ev_step = nullptr, ev_out[kHostChunks] = {nullptr}, ev_up[kHostChunks] = {nullptr};
    int rc = DARE_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&down, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_step, cudaEventDisableTiming);
    for (int c = 0; c < kHostChunks && e == cudaSuccess; c++) e = cudaEventCreateWithFlags(&ev_out[c], cudaEventDisableTiming);
    for (int c = 0; c < kHostChunks && e == cudaSuccess; c++) e = cudaEventCreateWithFlags(&ev_up[c], cudaEventDisableTiming);
    if (e != cudaSuccess) rc = check_cuda(ctx, e, "dare_timesteps_host: streams");
    dare_solve_report last{};
    for (int k = 0; k < nsteps && rc == DARE_OK; k++) {
        // the input of step k: slice c waits for the slice's result of step k - 1
        int nslices = 0;
        for (int c = 0; c < kHostChunks && e == cudaSuccess; c++) {
            const size_t off = (size_t)c * chunk;
            if (off >= total) break;
            const size_t len = off + chunk > total ? total - off : chunk;
            if (k > 0) e = cudaStreamWaitEvent(up, ev_out[c], 0);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dev + off, hb + off, len, cudaMemcpyHostToDevice, up);
            if (e == cudaSuccess) e = cudaEventRecord(ev_up[c], up);
            nslices = c + 1;
        }
        if (e != cudaSuccess) {
            rc = check_cuda(ctx, e, "dare_timesteps_host: upload");
            break;
        }
        dare_solve_report* rk = reps ? &reps[k] : &last;
        if (sliced) {
            // planes i .. i + 4 of the ghosted level (two ghost planes each
            // side) hold the stencil of internal plane i
            const int n0 = gd.n[0], og0 = gd.og[0];
            int done = 0;
            for (int c = 0; c < nslices && rc == DARE_OK; c++) {
                const size_t off = (size_t)c * chunk;
                const size_t len = off + chunk > total ? total - off : chunk;
                e = cudaStreamWaitEvent(ctx->stream, ev_up[c], 0);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(dev_old + off, dev + off, len, cudaMemcpyDeviceToDevice, ctx->stream);
                if (e != cudaSuccess) {
                    rc = check_cuda(ctx, e, "dare_timesteps_host: old level");
                    break;
                }
                const int planes_in = c == nslices - 1 ? gd.gn[0] : (int)((off + len) / plane_bytes);
                int upto = planes_in - 2 - og0;
                if (upto > n0) upto = n0;
                if (upto < 0) upto = 0;
                if (c == nslices - 1) upto = n0;
                if (upto > done) {
                    rc = launch_assemble_planes(s, desc, f->level[0], f->level[1], done, upto);   // Trilinos::Build
                    done = upto;
                }
            }
            if (rc) break;
            if ((rc = solve_and_copy_back(s, f, p, rk))) break;
            if (k == nsteps - 1 && (rc = dare_field_copy_to_old(f))) break;   // the next upload sets it otherwise
        } else {
            if ((e = cudaEventRecord(ev_in, up)) == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ev_in, 0);
            if (e != cudaSuccess) {
                rc = check_cuda(ctx, e, "dare_timesteps_host: upload");
                break;
            }
            if ((rc = dare_field_copy_to_old(f))) break;
            if ((rc = dare_timestep(s, f, desc, p, rk))) break;
        }
        // its result, slice by slice
        e = cudaEventRecord(ev_step, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(down, ev_step, 0);
        for (int c = 0; c < kHostChunks && e == cudaSuccess; c++) {
            const size_t off = (size_t)c * chunk;
            if (off >= total) break;
            const size_t len = off + chunk > total ? total - off : chunk;
            e = cudaMemcpyAsync(hb + off, dev + off, len, cudaMemcpyDeviceToHost, down);
            if (e == cudaSuccess) e = cudaEventRecord(ev_out[c], down);
        }
        if (e != cudaSuccess) rc = check_cuda(ctx, e, "dare_timesteps_host: download");
    }
    // the last result is on the host before returning (also after an error)
    if (down) cudaStreamSynchronize(down);
    if (up) cudaStreamSynchronize(up);
    for (auto& ev : ev_out)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : ev_up)
        if (ev) cudaEventDestroy(ev);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_step) cudaEventDestroy(ev_step);
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
    return rc;
}

int dare_ctx_set_profiling(dare_ctx* ctx, int on) {
    if (!ctx) return DARE_ERR_BAD_ARG;
    if (on) {
        for (auto& e : ctx->ev)
            if (!e) DARE_CUDA(ctx, cudaEventCreate(&e));
    }
    ctx->profiling = on ? 1 : 0;
    return DARE_OK;
}

int dare_ctx_reset_kernel_stats(dare_ctx* ctx) {
    if (!ctx) return DARE_ERR_BAD_ARG;
    std::memset(ctx->stat_ms, 0, sizeof(ctx->stat_ms));
    std::memset(ctx->stat_n, 0, sizeof(ctx->stat_n));
    return DARE_OK;
}

int dare_ctx_kernel_stats(const dare_ctx* ctx, int kernel_id, double* total_ms, int64_t* count) {
    if (!ctx || kernel_id < 0 || kernel_id >= KID_COUNT || !total_ms || !count) return DARE_ERR_BAD_ARG;
    *total_ms = ctx->stat_ms[kernel_id];
    *count = ctx->stat_n[kernel_id];
    return DARE_OK;
}

int dare_ctx_timer_start(dare_ctx* ctx) {
    if (!ctx) return DARE_ERR_BAD_ARG;
    if (!ctx->ev[14]) {
        DARE_CUDA(ctx, cudaEventCreate(&ctx->ev[14]));
        DARE_CUDA(ctx, cudaEventCreate(&ctx->ev[15]));
    }
    DARE_CUDA(ctx, cudaEventRecord(ctx->ev[14], ctx->stream));
    return DARE_OK;
}

int dare_ctx_timer_stop(dare_ctx* ctx, double* ms) {
    if (!ctx || !ms || !ctx->ev[14]) return DARE_ERR_BAD_ARG;
    DARE_CUDA(ctx, cudaEventRecord(ctx->ev[15], ctx->stream));
    DARE_CUDA(ctx, cudaEventSynchronize(ctx->ev[15]));
    float f = 0.f;
    DARE_CUDA(ctx, cudaEventElapsedTime(&f, ctx->ev[14], ctx->ev[15]));
    *ms = f;
    return DARE_OK;
}

}  // extern "C"
