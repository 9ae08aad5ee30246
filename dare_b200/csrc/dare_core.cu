// dare_core.cu -- context, grid, field and system management, halo fill,
// copies, CSR export.  See include/dare_gpu.h for the API contract.
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "dare_internal.cuh"

using namespace dare_gpu;

namespace dare_gpu {

int set_error(dare_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

int check_cuda(dare_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return set_error(ctx, e == cudaErrorMemoryAllocation ? DARE_ERR_OOM : DARE_ERR_CUDA, m);
}

// ---- kernels ---------------------------------------------------------------

// Periodic face-ghost fill along dimension d (HaloBuffer self-exchange on one
// rank; only ghosts outside the internal range in exactly this dimension).
__global__ void k_halo_fill(GridDev g, int d, double* __restrict__ phi) {
    const int e1 = d == 0 ? 1 : 0;
    const int e2 = d == 2 ? 1 : 2;
    const int64_t n1 = g.n[e1], n2 = g.n[e2];
    const int64_t total = (int64_t)2 * g.ng * n1 * n2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t % n2;
        const int64_t a = (t / n2) % n1;
        const int64_t layer = t / (n1 * n2);          // 0 .. 2*ng-1
        int ind[3], src[3];
        ind[e1] = (int)a + g.og[e1];
        ind[e2] = (int)b + g.og[e2];
        if (layer < g.ng) {                            // lower ghosts take the upper image
            ind[d] = (int)layer;
            src[d] = ind[d] + g.n[d];
        } else {                                        // upper ghosts take the lower image
            ind[d] = g.og[d] + g.n[d] + (int)(layer - g.ng);
            src[d] = ind[d] - g.n[d];
        }
        src[e1] = ind[e1];
        src[e2] = ind[e2];
        const int64_t o = ((int64_t)ind[0] * g.gn[1] + ind[1]) * g.gn[2] + ind[2];
        const int64_t s = ((int64_t)src[0] * g.gn[1] + src[1]) * g.gn[2] + src[2];
        phi[o] = phi[s];
    }
}

// x (internal) -> field (ghosted): Trilinos::CopyTo
__global__ void k_scatter_to_field(GridDev g, const double* __restrict__ x, double* __restrict__ phi) {
    const int64_t nyz = (int64_t)g.n[1] * g.n[2];
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g.ncell;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c / nyz);
        const int j = (int)((c / g.n[2]) % g.n[1]);
        const int k = (int)(c % g.n[2]);
        phi[local_index(g, i, j, k)] = x[c];
    }
}

// The end of a solve and the two calls after it in one pass: x = invd .* x
// (applyRightPrec, skipped when invd is null), CopyTo into the field, and
// the periodic face ghosts of ExchangeHaloCells, each ghost written by the
// internal cell it images (internal index q < ng: the upper ghost og + n + q;
// q >= n - ng: the lower ghost q - n + ng).  The values and the cells
// written are those of k_scale, k_scatter_to_field and k_halo_fill in turn
// (needs og[d] == ng and n[d] >= ng on the periodic dimensions).  Threads
// run along k, block rows along (i, j), without 64-bit divisions.
__global__ void k_solution_to_field(GridDev g, const double* __restrict__ invd, double* __restrict__ x,
                                    double* __restrict__ phi) {
    const int n1 = g.n[1], n2 = g.n[2];
    const int64_t rows = (int64_t)g.n[0] * n1;
    const int64_t rstep = (int64_t)gridDim.x * blockDim.y;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.y + threadIdx.y; r < rows; r += rstep) {
        const int i = (int)(r / n1), j = (int)(r - (int64_t)i * n1);
        const int64_t c0 = r * n2;
        for (int k = threadIdx.x; k < n2; k += blockDim.x) {
            const int64_t c = c0 + k;
            double v = x[c];
            if (invd) {
                v = invd[c] * v;
                x[c] = v;
            }
            const int q[3] = {i, j, k};
            const int ind[3] = {i + g.og[0], j + g.og[1], k + g.og[2]};
            phi[((int64_t)ind[0] * g.gn[1] + ind[1]) * g.gn[2] + ind[2]] = v;
            for (int d = 0; d < g.dim; d++) {
                if (!g.periodic[d]) continue;
                int t[3] = {ind[0], ind[1], ind[2]};
                if (q[d] < g.ng) {
                    t[d] = g.og[d] + g.n[d] + q[d];
                    phi[((int64_t)t[0] * g.gn[1] + t[1]) * g.gn[2] + t[2]] = v;
                }
                if (q[d] >= g.n[d] - g.ng) {
                    t[d] = q[d] - g.n[d] + g.ng;
                    phi[((int64_t)t[0] * g.gn[1] + t[1]) * g.gn[2] + t[2]] = v;
                }
            }
        }
    }
}

// field (ghosted) -> x (internal): the initial guess of BuildNew
__global__ void k_gather_from_field(GridDev g, const double* __restrict__ phi, double* __restrict__ x) {
    const int64_t nyz = (int64_t)g.n[1] * g.n[2];
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g.ncell;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c / nyz);
        const int j = (int)((c / g.n[2]) % g.n[1]);
        const int k = (int)(c % g.n[2]);
        x[c] = phi[local_index(g, i, j, k)];
    }
}

// Linear interpolation of cell values to faces (Interpolation_Cartesian.h:139-158,
// Divide<2> = multiply by 1/2, Math/Divisors.h:71-79).
__global__ void k_face_average(GridDev g, int d, const double* __restrict__ cell, double* __restrict__ face) {
    int nf[3] = {g.n[0], g.n[1], g.n[2]};
    nf[d] += 1;
    const int64_t total = (int64_t)nf[0] * nf[1] * nf[2];
    const int64_t cs[3] = {(int64_t)g.n[1] * g.n[2], g.n[2], 1};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int idx[3];
        idx[2] = (int)(t % nf[2]);
        idx[1] = (int)((t / nf[2]) % nf[1]);
        idx[0] = (int)(t / ((int64_t)nf[1] * nf[2]));
        int lo = idx[d] - 1, hi = idx[d];
        if (lo < 0) lo = g.periodic[d] ? g.n[d] - 1 : 0;
        if (hi >= g.n[d]) hi = g.periodic[d] ? 0 : g.n[d] - 1;
        int a[3] = {idx[0], idx[1], idx[2]}, b[3] = {idx[0], idx[1], idx[2]};
        a[d] = lo;
        b[d] = hi;
        const double va = cell[a[0] * cs[0] + a[1] * cs[1] + a[2]];
        const double vb = cell[b[0] * cs[0] + b[1] * cs[1] + b[2]];
        face[t] = (va + vb) * (1. / 2.);
    }
}

int launch_gather(dare_ctx* ctx, const GridDev& g, const double* phi, double* x) {
    int blocks = grid_blocks(ctx, g.ncell, 256, 8);
    k_gather_from_field<<<blocks, 256, 0, ctx->stream>>>(g, phi, x);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

int launch_scatter(dare_ctx* ctx, const GridDev& g, const double* x, double* phi) {
    int blocks = grid_blocks(ctx, g.ncell, 256, 8);
    k_scatter_to_field<<<blocks, 256, 0, ctx->stream>>>(g, x, phi);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

bool solution_to_field_ok(const GridDev& g) {
    for (int d = 0; d < g.dim; d++)
        if (g.periodic[d] && (g.og[d] != g.ng || g.n[d] < g.ng)) return false;
    return g.ncell > 0;
}

// Block shape of k_solution_to_field: threads along k up to 256 (a power of
// two covering n2), the rest of the 256 along the rows.
dim3 solution_to_field_block(const GridDev& g) {
    int bx = 1;
    while (bx < g.n[2] && bx < 256) bx *= 2;
    return dim3(bx, 256 / bx, 1);
}

int launch_solution_to_field(dare_ctx* ctx, const GridDev& g, const double* invd, double* x, double* phi) {
    if (!solution_to_field_ok(g)) return set_error(ctx, DARE_ERR_BAD_ARG, "solution_to_field: ghost layout");
    const dim3 block = solution_to_field_block(g);
    const int64_t rows = (int64_t)g.n[0] * g.n[1];
    const int blocks = grid_blocks(ctx, rows, (int)block.y, 8);
    k_solution_to_field<<<blocks, block, 0, ctx->stream>>>(g, invd, x, phi);
    DARE_LAUNCHED(ctx);
    return DARE_OK;
}

int launch_halo(dare_ctx* ctx, const GridDev& g, double* phi) {
    for (int d = 0; d < g.dim; d++) {
        if (!g.periodic[d]) continue;
        const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
        const int64_t total = (int64_t)2 * g.ng * g.n[e1] * g.n[e2];
        int blocks = grid_blocks(ctx, total, 256, 8);
        k_halo_fill<<<blocks, 256, 0, ctx->stream>>>(g, d, phi);
        DARE_LAUNCHED(ctx);
    }
    return DARE_OK;
}

}  // namespace dare_gpu

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

int dare_ctx_create(int device, dare_ctx** out) {
    if (!out) return DARE_ERR_BAD_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return DARE_ERR_CUDA;
    }
    dare_ctx* ctx = new (std::nothrow) dare_ctx();
    if (!ctx) return DARE_ERR_OOM;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return DARE_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return DARE_OK;
}

int dare_ctx_destroy(dare_ctx* ctx) {
    if (!ctx) return DARE_ERR_BAD_ARG;
    cudaSetDevice(ctx->device);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return DARE_OK;
}

int dare_ctx_set_stream(dare_ctx* ctx, void* stream) {
    if (!ctx) return DARE_ERR_BAD_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return DARE_OK;
}

void* dare_ctx_get_stream(dare_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int dare_ctx_synchronize(dare_ctx* ctx) {
    if (!ctx) return DARE_ERR_BAD_ARG;
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

const char* dare_ctx_last_error(const dare_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int64_t dare_ctx_launch_count(const dare_ctx* ctx) { return ctx ? ctx->launches : -1; }

int dare_grid_create_staggered(dare_ctx* ctx, int dim, const int64_t n[3], const double size[3], int num_ghost,
                               const int periodic[3], const int staggered[3], dare_grid** out) {
    if (!ctx || !out || !n || !size || dim < 1 || dim > 3 || num_ghost < 2)
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_grid_create: bad arguments (dim 1..3, num_ghost >= 2)");
    *out = nullptr;
    GridDev g{};
    g.dim = dim;
    g.ng = num_ghost;
    int64_t total = 1, total_g = 1;
    for (int d = 0; d < 3; d++) {
        const bool active = d < dim;
        const int64_t nb = active ? n[d] : 1;
        // CartesianMesh.inl:60-69: resolution must exceed the ghost count
        if (active && (nb <= num_ghost || nb > (1 << 30)))
            return set_error(ctx, DARE_ERR_BAD_ARG, "dare_grid_create: resolution must be > num_ghost");
        g.periodic[d] = active && periodic ? (periodic[d] != 0) : 0;
        // CartesianRepresentation.inl:67-76: a staggered direction gains the
        // cell at its upper end, on non-periodic grids only
        g.staggered[d] = active && staggered ? (staggered[d] != 0) : 0;
        const int64_t nd = nb + (g.staggered[d] && !g.periodic[d] ? 1 : 0);
        g.n[d] = (int)nd;
        g.og[d] = active ? num_ghost : 0;
        g.gn[d] = (int)(nd + 2 * g.og[d]);
        total *= nd;
        total_g *= g.gn[d];
    }
    if (total_g >= ((int64_t)1 << 31))
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_grid_create: grid exceeds 2^31 ghosted cells");
    g.ncell = total;
    g.ncell_ghosted = total_g;
    // CartesianMesh.inl:75-83: the cell width of the base grid
    double vol = 1.;
    for (int d = 0; d < 3; d++) g.dx[d] = 1.;
    for (int d = 0; d < dim; d++) g.dx[d] = size[d] / (double)n[d];
    for (int d = 0; d < dim; d++) vol *= g.dx[d];
    for (int d = 0; d < 3; d++) g.area[d] = d < dim ? vol / g.dx[d] : 0.;
    g.volume = vol;
    for (int d = 0; d < 3; d++) g.origin[d] = g.staggered[d] && !g.periodic[d] ? -g.dx[d] * 0.5 : 0.;
    dare_grid* gr = new (std::nothrow) dare_grid();
    if (!gr) return DARE_ERR_OOM;
    gr->ctx = ctx;
    gr->dev = g;
    *out = gr;
    return DARE_OK;
}

int dare_grid_create(dare_ctx* ctx, int dim, const int64_t n[3], const double size[3], int num_ghost,
                     const int periodic[3], dare_grid** out) {
    return dare_grid_create_staggered(ctx, dim, n, size, num_ghost, periodic, nullptr, out);
}

int dare_grid_destroy(dare_grid* g) {
    delete g;
    return DARE_OK;
}

int dare_grid_get_info(const dare_grid* g, dare_grid_info* info) {
    if (!g || !info) return DARE_ERR_BAD_ARG;
    const GridDev& d = g->dev;
    info->dim = d.dim;
    info->num_ghost = d.ng;
    for (int i = 0; i < 3; i++) {
        info->n[i] = d.n[i];
        info->n_ghosted[i] = d.gn[i];
        info->dx[i] = d.dx[i];
        info->area[i] = d.area[i];
        info->periodic[i] = d.periodic[i];
        info->staggered[i] = d.staggered[i];
        info->origin[i] = d.origin[i];
    }
    info->num_cells = d.ncell;
    info->num_cells_ghosted = d.ncell_ghosted;
    info->volume = d.volume;
    return DARE_OK;
}

int dare_field_create(dare_grid* g, int num_levels, dare_field** out) {
    return dare_field_create_n(g, num_levels, 1, out);
}

int dare_field_create_n(dare_grid* g, int num_levels, int num_components, dare_field** out) {
    if (!g || !out || num_levels < 1 || num_levels > 8 || num_components < 1 || num_components > 64)
        return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = g->ctx;
    *out = nullptr;
    dare_field* f = new (std::nothrow) dare_field();
    if (!f) return DARE_ERR_OOM;
    f->grid = g;
    f->device = ctx->device;
    f->num_levels = num_levels;
    f->ncomp = num_components;
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)g->dev.ncell_ghosted * num_components * sizeof(double);
    for (int l = 0; l < num_levels; l++) {
        cudaError_t e = cudaMalloc(&f->level[l], bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(f->level[l], 0, bytes, ctx->stream);
        if (e != cudaSuccess) {
            for (int m = 0; m <= l; m++) cudaFree(f->level[m]);
            delete f;
            return check_cuda(ctx, e, "dare_field_create");
        }
    }
    *out = f;
    return DARE_OK;
}

int dare_field_destroy(dare_field* f) {
    if (!f) return DARE_ERR_BAD_ARG;
    cudaSetDevice(f->device);
    for (int l = 0; l < f->num_levels; l++) cudaFree(f->level[l]);
    delete f;
    return DARE_OK;
}

// The host side of a field or system uses the reference's interleaved order
// (GridVector.inl:68-71: data[cell * N + c]); the device keeps each component
// contiguous.  These convert between the two through a host buffer.
static void interleave(const double* comp_major, int64_t n, int ncomp, double* inter) {
    for (int64_t i = 0; i < n; i++)
        for (int c = 0; c < ncomp; c++) inter[i * ncomp + c] = comp_major[(int64_t)c * n + i];
}
static void deinterleave(const double* inter, int64_t n, int ncomp, double* comp_major) {
    for (int c = 0; c < ncomp; c++)
        for (int64_t i = 0; i < n; i++) comp_major[(int64_t)c * n + i] = inter[i * ncomp + c];
}

static int upload_interleaved(dare_ctx* ctx, double* dev, const double* host, int64_t n, int ncomp) {
    if (ncomp == 1) {
        DARE_CUDA(ctx, cudaMemcpyAsync(dev, host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    } else {
        std::vector<double> t((size_t)n * ncomp);
        deinterleave(host, n, ncomp, t.data());
        DARE_CUDA(ctx, cudaMemcpyAsync(dev, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return DARE_OK;
}

static int download_interleaved(dare_ctx* ctx, double* host, const double* dev, int64_t n, int ncomp) {
    if (ncomp == 1) {
        DARE_CUDA(ctx, cudaMemcpyAsync(host, dev, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    } else {
        std::vector<double> t((size_t)n * ncomp);
        DARE_CUDA(ctx, cudaMemcpyAsync(t.data(), dev, t.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        interleave(t.data(), n, ncomp, host);
    }
    return DARE_OK;
}

int dare_field_upload(dare_field* f, int level, const double* host) {
    if (!f || !host || level < 0 || level >= f->num_levels) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = f->grid->ctx;
    int rc = upload_interleaved(ctx, f->level[level], host, f->grid->dev.ncell_ghosted, f->ncomp);
    if (rc) return rc;
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_field_download(dare_field* f, int level, double* host) {
    if (!f || !host || level < 0 || level >= f->num_levels) return DARE_ERR_BAD_ARG;
    return download_interleaved(f->grid->ctx, host, f->level[level], f->grid->dev.ncell_ghosted, f->ncomp);
}

int dare_field_num_components(const dare_field* f) { return f ? f->ncomp : DARE_ERR_BAD_ARG; }

double* dare_field_device_ptr(dare_field* f, int level) {
    if (!f || level < 0 || level >= f->num_levels) return nullptr;
    return f->level[level];
}

int dare_field_exchange_halo(dare_field* f) {
    if (!f) return DARE_ERR_BAD_ARG;
    for (int c = 0; c < f->ncomp; c++) {
        const int rc = launch_halo(f->grid->ctx, f->grid->dev, f->level[0] + (size_t)c * f->grid->dev.ncell_ghosted);
        if (rc) return rc;
    }
    return DARE_OK;
}

int dare_field_copy_to_old(dare_field* f) {
    if (!f) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = f->grid->ctx;
    const size_t bytes = (size_t)f->grid->dev.ncell_ghosted * f->ncomp * sizeof(double);
    for (int n = f->num_levels - 1; n > 0; n--)
        DARE_CUDA(ctx, cudaMemcpyAsync(f->level[n], f->level[n - 1], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return DARE_OK;
}

int dare_system_create(dare_grid* g, dare_system** out) { return dare_system_create_n(g, 1, out); }

int dare_system_create_n(dare_grid* g, int num_components, dare_system** out) {
    if (!g || !out || num_components < 1 || num_components > 64) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = g->ctx;
    *out = nullptr;
    if ((int64_t)g->dev.n[0] * num_components >= ((int64_t)1 << 30) ||
        g->dev.ncell_ghosted * num_components >= ((int64_t)1 << 31))
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_system_create: too many cells x components");
    dare_system* s = new (std::nothrow) dare_system();
    if (!s) return DARE_ERR_OOM;
    s->grid = g;
    s->device = ctx->device;
    s->ncomp = num_components;
    s->sdev = g->dev;
    s->sdev.ncomp = num_components;
    s->sdev.n[0] = g->dev.n[0] * num_components;
    s->sdev.ncell = g->dev.ncell * num_components;
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)s->sdev.ncell;
    cudaError_t e = cudaMalloc(&s->diag, n * kSlots * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s->rhs, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s->x, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->diag, 0, n * kSlots * sizeof(double), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->rhs, 0, n * sizeof(double), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->x, 0, n * sizeof(double), ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(s->diag);
        cudaFree(s->rhs);
        cudaFree(s->x);
        delete s;
        return check_cuda(ctx, e, "dare_system_create");
    }
    // non-periodic faces default to homogeneous Neumann
    for (int d = 0; d < 3; d++) {
        const int t = (d < g->dev.dim && !g->dev.periodic[d]) ? DARE_BC_NEUMANN : DARE_BC_PERIODIC;
        s->bc_type[2 * d] = s->bc_type[2 * d + 1] = t;
    }
    *out = s;
    return DARE_OK;
}

int dare_system_destroy(dare_system* s) {
    if (!s) return DARE_ERR_BAD_ARG;
    cudaSetDevice(s->device);
    dare_solver_ws_free(s->ws);
    cudaFree(s->diag);
    cudaFree(s->rhs);
    cudaFree(s->x);
    delete s;
    return DARE_OK;
}

int dare_system_set_bc(dare_system* s, int face, int type, double value) {
    if (!s || face < DARE_WEST || face > DARE_TOP) return DARE_ERR_BAD_ARG;
    const GridDev& g = s->grid->dev;
    const int d = (face - 1) / 2;
    if (d >= g.dim) return set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "dare_system_set_bc: inactive dimension");
    if (g.periodic[d]) {
        if (type != DARE_BC_PERIODIC)
            return set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "dare_system_set_bc: dimension is periodic");
    } else if (type != DARE_BC_DIRICHLET && type != DARE_BC_NEUMANN) {
        return set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "dare_system_set_bc: non-periodic face needs Dirichlet or Neumann");
    }
    s->bc_type[face - 1] = type;
    s->bc_value[face - 1] = value;
    for (int c = 0; c < (int)s->bc_type_c.size() / 6; c++) {   // every component
        s->bc_type_c[c * 6 + face - 1] = type;
        s->bc_value_c[c * 6 + face - 1] = value;
    }
    return DARE_OK;
}

int dare_system_set_bc_component(dare_system* s, int component, int face, int type, double value) {
    if (!s || face < DARE_WEST || face > DARE_TOP) return DARE_ERR_BAD_ARG;
    if (component < 0) return dare_system_set_bc(s, face, type, value);
    if (component >= s->ncomp)
        return set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "dare_system_set_bc_component: no such component");
    const GridDev& g = s->grid->dev;
    const int d = (face - 1) / 2;
    if (d >= g.dim) return set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "dare_system_set_bc_component: inactive dimension");
    if (g.periodic[d]) {
        if (type != DARE_BC_PERIODIC)
            return set_error(s->grid->ctx, DARE_ERR_BAD_ARG, "dare_system_set_bc_component: dimension is periodic");
    } else if (type != DARE_BC_DIRICHLET && type != DARE_BC_NEUMANN) {
        return set_error(s->grid->ctx, DARE_ERR_BAD_ARG,
                         "dare_system_set_bc_component: non-periodic face needs Dirichlet or Neumann");
    }
    if (s->bc_type_c.empty()) {   // start from the whole-system conditions
        s->bc_type_c.resize((size_t)s->ncomp * 6);
        s->bc_value_c.resize((size_t)s->ncomp * 6);
        for (int c = 0; c < s->ncomp; c++)
            for (int f = 0; f < 6; f++) {
                s->bc_type_c[c * 6 + f] = s->bc_type[f];
                s->bc_value_c[c * 6 + f] = s->bc_value[f];
            }
    }
    s->bc_type_c[(size_t)component * 6 + face - 1] = type;
    s->bc_value_c[(size_t)component * 6 + face - 1] = value;
    return DARE_OK;
}

int dare_system_set_coefficients(dare_system* s, const double* diag7, const double* rhs, const double* x0) {
    if (!s) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = s->grid->ctx;
    const int64_t n = s->grid->dev.ncell;
    const int nc = s->ncomp;
    int rc;
    if (diag7)
        for (int q = 0; q < kSlots; q++)
            if ((rc = upload_interleaved(ctx, s->diag + (size_t)q * n * nc, diag7 + (size_t)q * n * nc, n, nc))) return rc;
    if (rhs && (rc = upload_interleaved(ctx, s->rhs, rhs, n, nc))) return rc;
    if (x0 && (rc = upload_interleaved(ctx, s->x, x0, n, nc))) return rc;
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_system_get_coefficients(dare_system* s, double* diag7, double* rhs) {
    if (!s) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = s->grid->ctx;
    const int64_t n = s->grid->dev.ncell;
    const int nc = s->ncomp;
    int rc;
    if (diag7)
        for (int q = 0; q < kSlots; q++)
            if ((rc = download_interleaved(ctx, diag7 + (size_t)q * n * nc, s->diag + (size_t)q * n * nc, n, nc)))
                return rc;
    if (rhs && (rc = download_interleaved(ctx, rhs, s->rhs, n, nc))) return rc;
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DARE_OK;
}

int dare_system_set_initial_guess(dare_system* s, const double* x0) {
    return dare_system_set_coefficients(s, nullptr, nullptr, x0);
}

int dare_system_get_solution(dare_system* s, double* x) {
    if (!s || !x) return DARE_ERR_BAD_ARG;
    return download_interleaved(s->grid->ctx, x, s->x, s->grid->dev.ncell, s->ncomp);
}

int dare_system_num_components(const dare_system* s) { return s ? s->ncomp : DARE_ERR_BAD_ARG; }

double* dare_system_device_ptr(dare_system* s, int which) {
    if (!s) return nullptr;
    if (which >= 0 && which < kSlots) return s->diag + (size_t)which * s->sdev.ncell;
    if (which == 7) return s->rhs;
    if (which == 8) return s->x;
    return nullptr;
}

// Pattern of a row: all slots of active dimensions, minus the neighbours
// removed at non-periodic boundaries (the Remove() calls of the BC folding).
static unsigned row_mask(const GridDev& g, int i, int j, int k) {
    unsigned m = 1;
    const int idx[3] = {i, j, k};
    for (int d = 0; d < g.dim; d++) {
        const unsigned lo = 1u << (2 * d + 1), hi = 1u << (2 * d + 2);
        m |= lo | hi;
        if (!g.periodic[d]) {
            if (idx[d] == 0) m &= ~lo;
            if (idx[d] == g.n[d] - 1) m &= ~hi;
        }
    }
    return m;
}

int64_t dare_system_csr_nnz(dare_system* s) {
    if (!s) return -1;
    const GridDev& g = s->grid->dev;
    int64_t nnz = 0;
    for (int i = 0; i < g.n[0]; i++)
        for (int j = 0; j < g.n[1]; j++)
            for (int k = 0; k < g.n[2]; k++) nnz += __builtin_popcount(row_mask(g, i, j, k));
    return nnz * s->ncomp;
}

int dare_system_export_csr(dare_system* s, int64_t* rowptr, int64_t* cols, double* vals) {
    if (!s || !rowptr || !cols || !vals) return DARE_ERR_BAD_ARG;
    const GridDev& g = s->grid->dev;
    const int nc = s->ncomp;
    std::vector<double> diag((size_t)g.ncell * nc * kSlots);   // interleaved rows: cell * N + c
    int rc = dare_system_get_coefficients(s, diag.data(), nullptr);
    if (rc) return rc;
    static const int emit_order[7] = {DARE_WEST, DARE_SOUTH, DARE_BOTTOM, DARE_CENTER, DARE_TOP, DARE_NORTH, DARE_EAST};
    int64_t pos = 0;
    rowptr[0] = 0;
    for (int i = 0; i < g.n[0]; i++)
        for (int j = 0; j < g.n[1]; j++)
            for (int k = 0; k < g.n[2]; k++) {
                const int64_t cell = ((int64_t)i * g.n[1] + j) * g.n[2] + k;
                const unsigned m = row_mask(g, i, j, k);
                int64_t nb[7];
                neighbour_ordinals(g, i, j, k, cell, nb);
                // MatrixBlock::Finalize per component: column = neighbour * N + c
                // (MatrixBlock_Cartesian.inl:127-240), rows cell * N + c
                for (int comp = 0; comp < nc; comp++) {
                const int64_t c = cell * nc + comp;
                int64_t rc_[7];
                double rv[7];
                int cnt = 0;
                for (int e = 0; e < 7; e++) {
                    const int p = emit_order[e];
                    if (!(m & (1u << p))) continue;
                    rc_[cnt] = nb[p] * nc + comp;
                    rv[cnt] = diag[(size_t)p * g.ncell * nc + c];
                    cnt++;
                }
                for (int a = 1; a < cnt; a++) {        // sort by column
                    int64_t kc = rc_[a];
                    double kv = rv[a];
                    int b = a - 1;
                    while (b >= 0 && rc_[b] > kc) {
                        rc_[b + 1] = rc_[b];
                        rv[b + 1] = rv[b];
                        b--;
                    }
                    rc_[b + 1] = kc;
                    rv[b + 1] = kv;
                }
                for (int e = 0; e < cnt; e++) {
                    cols[pos] = rc_[e];
                    vals[pos] = rv[e];
                    pos++;
                }
                rowptr[c + 1] = pos;
                }
            }
    return DARE_OK;
}

int dare_system_copy_to(dare_system* s, dare_field* f) {
    if (!s || !f || f->grid != s->grid || f->ncomp != s->ncomp) return DARE_ERR_BAD_ARG;
    const GridDev& g = s->grid->dev;
    for (int c = 0; c < s->ncomp; c++) {
        const int rc = launch_scatter(s->grid->ctx, g, s->x + (size_t)c * g.ncell, f->level[0] + (size_t)c * g.ncell_ghosted);
        if (rc) return rc;
    }
    return DARE_OK;
}

int dare_face_average(dare_grid* gr, const double* cell_D, double* face_D[3]) {
    if (!gr || !cell_D || !face_D) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = gr->ctx;
    const GridDev& g = gr->dev;
    for (int d = 0; d < g.dim; d++) {
        if (!face_D[d]) return DARE_ERR_BAD_ARG;
        int64_t total = g.ncell / g.n[d] * (g.n[d] + 1);
        int blocks = grid_blocks(ctx, total, 256, 8);
        k_face_average<<<blocks, 256, 0, ctx->stream>>>(g, d, cell_D, face_D[d]);
        DARE_LAUNCHED(ctx);
    }
    return DARE_OK;
}

}  // extern "C"
