// dare_slabs.cu -- the implicit step on slabs of i-planes: the reference's
// distribution of a Cartesian grid over ranks
// (Grid/Cartesian/CartesianDistribution.h:94-380) with its halo exchange
// (MPI/HaloBuffer.inl:30-208) and the reductions of a distributed
// BiCGStab2 (every dot product of BiCGStab2.inl:339-559 summed over ranks).
//
// A slab owns planes [i0, i1) of the grid: its own field (ghosted, every
// time level), its own system rows and its own solver vectors, exactly the
// storage a rank would hold.  Three exchange points connect the slabs:
//   * before an assembly, `ng` boundary planes of the field go into the
//     neighbours' ghost planes (the van Leer face of cell i reads i - 2);
//   * before every marching kernel, one boundary plane of each SpMV operand
//     input goes into the neighbour's halo buffer, which the kernel reads as
//     the plane before its first (after its last) plane;
//   * every reduction sums the partials of all slabs' work items: a slab's
//     items write their own range of slots and the last item to arrive, in
//     whichever slab, sums all slots in slot order.
// On one device each plane crosses with one cudaMemcpyAsync and the scalar
// state is one shared SolverState.  Over several GPUs the copies become
// ncclSend / ncclRecv pairs between neighbouring ranks (the same bytes in the
// same order) and the reduction an all-reduce of each rank's packed partials
// before its last kernel evaluates the scalar step.
//
// The slabs' coefficients are the global assembly's rows bit for bit (the
// same kernel sees the same values); the solve differs from the single-grid
// solve only in the order of the partial sums (rounding).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "dare_march.cuh"

using namespace dare_gpu;

namespace dare_gpu {
int launch_assemble(dare_system* s, const dare_assembly_desc* desc, const double* phi, const double* phi_old);
}  // namespace dare_gpu

constexpr int kMaxSlabs = 8;

struct dare_slabs {
    dare_ctx* ctx = nullptr;
    int device = 0;                  // for dare_slabs_destroy, which does not touch ctx
    GridDev global{};
    int ncomp = 1;                   // field components (stacked along i in the solver's vectors)
    int S = 0;
    int periodic_x = 0;
    std::vector<int> i0, i1;
    std::vector<dare_grid*> grids;
    std::vector<dare_field*> fields;
    std::vector<dare_system*> systems;
    // solver: per-slab work decomposition, shared reduction slots and state
    std::vector<MarchCfg> march;
    std::vector<int> item_base, sblocks, sblock_base;
    int items_total = 0, sblocks_total = 0;
    double* halo = nullptr;          // per slab: [2 operand inputs][2 sides][component][one plane]
    double* partials = nullptr;      // kMaxQ * kMaxBlocks (+ one scratch value)
    SolverState* st = nullptr;
    SolverState* st_host = nullptr;  // pinned
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // two iterations, plain / Jacobi
};

namespace {

int lower(const dare_slabs* sl, int s) { return s > 0 ? s - 1 : (sl->periodic_x ? sl->S - 1 : -1); }
int upper(const dare_slabs* sl, int s) { return s < sl->S - 1 ? s + 1 : (sl->periodic_x ? 0 : -1); }

int64_t plane_cells(const dare_slabs* sl) { return (int64_t)sl->global.n[1] * sl->global.n[2]; }
int64_t ghosted_plane(const dare_slabs* sl) { return (int64_t)sl->global.gn[1] * sl->global.gn[2]; }

double* halo_buf(dare_slabs* sl, int s, int z, int side) {
    return sl->halo + ((size_t)(s * 2 + z) * 2 + side) * (size_t)sl->ncomp * plane_cells(sl);
}

// The transfer primitive of the slab path: `count` runs of `bytes` from slab
// memory to slab memory (runs `src_pitch` / `dst_pitch` bytes apart: one run
// per field component), in stream order.
int transfer(dare_ctx* ctx, void* dst, const void* src, size_t bytes, int count = 1, size_t dst_pitch = 0,
             size_t src_pitch = 0) {
    for (int c = 0; c < count; c++)
        DARE_CUDA(ctx, cudaMemcpyAsync(static_cast<char*>(dst) + c * dst_pitch,
                                       static_cast<const char*>(src) + c * src_pitch, bytes, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
    return DARE_OK;
}

// One marching kernel over every slab: the boundary planes of its operand
// inputs first go to the neighbours' halo buffers, then each slab runs its
// items, their partial sums in the slab's range of the shared slots.
template <class K>
int march_slabs(dare_slabs* sl, const std::vector<K>& ks) {
    using T = typename K::type;
    static_assert(sizeof(T) == sizeof(double), "the slab path runs in FP64");
    dare_ctx* ctx = sl->ctx;
    const int64_t P = plane_cells(sl);
    int rc;
    const int nc = sl->ncomp;
    const size_t pb = (size_t)P * sizeof(T);   // one plane
    for (int s = 0; s < sl->S; s++) {
        const int lo = lower(sl, s), hi = upper(sl, s);
        for (int z = 0; z < K::NZ; z++) {
            // each component's last plane of the lower neighbour, first plane of the upper one
            if (lo >= 0) {
                const int nl = sl->i1[lo] - sl->i0[lo];
                if ((rc = transfer(ctx, halo_buf(sl, s, z, 0), ks[lo].zs[z] + (int64_t)(nl - 1) * P, pb, nc, pb,
                                   (size_t)nl * pb)))
                    return rc;
            }
            if (hi >= 0) {
                const int nh = sl->i1[hi] - sl->i0[hi];
                if ((rc = transfer(ctx, halo_buf(sl, s, z, 1), ks[hi].zs[z], pb, nc, pb, (size_t)nh * pb))) return rc;
            }
        }
    }
    for (int s = 0; s < sl->S; s++) {
        MarchCfg m = sl->march[s];
        m.item_base = sl->item_base[s];
        m.nitems_total = sl->items_total;
        const int lo = lower(sl, s), hi = upper(sl, s);
        for (int z = 0; z < K::NZ; z++) {
            m.halo[z][0] = lo >= 0 ? halo_buf(sl, s, z, 0) : nullptr;
            m.halo[z][1] = hi >= 0 ? halo_buf(sl, s, z, 1) : nullptr;
        }
        if ((rc = launch_march<K, true>(ctx, sl->systems[s]->sdev, m, ks[s], sl->st, sl->partials))) return rc;
    }
    return DARE_OK;
}

struct SlabVecs {
    std::vector<VecsT<double>> vs;
    std::vector<OpT<double>> op;
};

SlabVecs slab_vectors(dare_slabs* sl, bool jacobi) {
    SlabVecs v;
    for (int s = 0; s < sl->S; s++) {
        dare_system* sy = sl->systems[s];
        const int64_t n = sy->sdev.ncell;
        v.vs.push_back(carve_vecs<double>(sy->ws->vec, n, sy->x, sy->rhs));
        v.op.push_back(jacobi ? OpT<double>{nullptr, sy->ws->ahat, n} : OpT<double>{sy->diag, sy->diag + n, n});
    }
    return v;
}

template <bool UNIT>
int slab_iteration(dare_slabs* sl, const SlabVecs& v) {
    const int S = sl->S;
    int rc;
    std::vector<FStep1<double, UNIT>> k1;
    std::vector<FStep2<double, UNIT>> k2;
    std::vector<FStep3<double, UNIT>> k3;
    std::vector<FStep4<double, UNIT>> k4;
    for (int s = 0; s < S; s++) {
        k1.push_back(make_step1<double, UNIT>(v.op[s], v.vs[s]));
        k2.push_back(make_step2<double, UNIT>(v.op[s], v.vs[s]));
        k3.push_back(make_step3<double, UNIT>(v.op[s], v.vs[s]));
        k4.push_back(make_step4<double, UNIT>(v.op[s], v.vs[s]));
    }
    if ((rc = march_slabs(sl, k1))) return rc;
    if ((rc = march_slabs(sl, k2))) return rc;
    if ((rc = march_slabs(sl, k3))) return rc;
    if ((rc = march_slabs(sl, k4))) return rc;
    for (int s = 0; s < S; s++) {
        const VecsT<double>& vs = v.vs[s];
        k_step5<double><<<sl->sblocks[s], 256, 0, sl->ctx->stream>>>(
            sl->systems[s]->sdev.ncell, vs.x, vs.r[0], vs.s[1], vs.t, vs.u[0], vs.u[1], vs.r[1], vs.v[1], vs.w, vs.rh,
            sl->st, sl->partials, sl->sblock_base[s], sl->sblocks_total, 0);
        DARE_LAUNCHED(sl->ctx);
    }
    return DARE_OK;
}

// Two iterations over every slab, captured as one CUDA graph.
template <bool UNIT>
int slab_graph(dare_slabs* sl, const SlabVecs& v, cudaGraphExec_t* out) {
    dare_ctx* ctx = sl->ctx;
    cudaStream_t cap;
    DARE_CUDA(ctx, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaStream_t saved = ctx->stream;
    ctx->stream = cap;
    cudaGraph_t graph = nullptr;
    int rc = DARE_OK;
    const int64_t launches0 = ctx->launches;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = slab_iteration<UNIT>(sl, v);
        if (rc == DARE_OK) rc = slab_iteration<UNIT>(sl, v);
        const cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
        if (e == cudaSuccess) e = e2;
    }
    ctx->stream = saved;
    ctx->launches = launches0;   // captured, not executed
    if (e == cudaSuccess && rc == DARE_OK) e = cudaGraphInstantiate(out, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != DARE_OK) return rc;
    if (e != cudaSuccess) return check_cuda(ctx, e, "slab graph capture");
    return DARE_OK;
}

// Iterations until the shared done flag is set (graph replays of two
// iterations, the state polled every few pairs).
template <bool UNIT>
int slab_run(dare_slabs* sl, const SlabVecs& v, int max_it, int check_every) {
    dare_ctx* ctx = sl->ctx;
    cudaGraphExec_t* ge = &sl->graph[UNIT ? 1 : 0];
    int rc;
    if (!*ge && (rc = slab_graph<UNIT>(sl, v, ge))) return rc;
    if (check_every <= 0) {
        const int64_t per = (int64_t)1 << 21;
        check_every = (int)std::min<int64_t>(8, std::max<int64_t>(1, (per + sl->global.ncell - 1) / sl->global.ncell));
    }
    const int launches_per_pair = 2 * (4 * sl->S + sl->S);
    const int max_pairs = max_it / 2 + 2;
    for (int gi = 0; gi < max_pairs; gi++) {
        DARE_CUDA(ctx, cudaGraphLaunch(*ge, ctx->stream));
        ctx->launches += launches_per_pair;
        if ((gi + 1) % check_every == 0 || gi + 1 == max_pairs) {
            DARE_CUDA(ctx, cudaMemcpyAsync(sl->st_host, sl->st, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                           ctx->stream));
            DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (sl->st_host->done) break;
        }
    }
    if (!sl->st_host->done) return set_error(ctx, DARE_ERR_STATE, "slab bicgstab2: iteration bound reached without a status");
    return DARE_OK;
}

int slab_scale(dare_slabs* sl) {
    for (int s = 0; s < sl->S; s++) {
        dare_system* sy = sl->systems[s];
        const int rc = launch_scale(sl->ctx, sy->sdev.ncell, sy->ws->invd, sy->x);
        if (rc) return rc;
    }
    return DARE_OK;
}

// ||b - A x|| over all slabs (the general operator, x in the slabs' systems)
int slab_true_residual(dare_slabs* sl, double* out_host) {
    std::vector<FResidual<double>> ks;
    double* dres = sl->partials + (size_t)kMaxQ * kMaxBlocks;
    for (int s = 0; s < sl->S; s++) {
        dare_system* sy = sl->systems[s];
        const int64_t n = sy->sdev.ncell;
        ks.push_back(make_residual(OpT<double>{sy->diag, sy->diag + n, n}, sy->x, sy->rhs, dres));
    }
    int rc = march_slabs(sl, ks);
    if (rc) return rc;
    DARE_CUDA(sl->ctx, cudaMemcpyAsync(out_host, dres, sizeof(double), cudaMemcpyDeviceToHost, sl->ctx->stream));
    DARE_CUDA(sl->ctx, cudaStreamSynchronize(sl->ctx->stream));
    return DARE_OK;
}

void slabs_free(dare_slabs* sl) {
    if (!sl) return;
    for (auto& g : sl->graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto* sy : sl->systems)
        if (sy) dare_system_destroy(sy);
    for (auto* f : sl->fields)
        if (f) dare_field_destroy(f);
    for (auto* g : sl->grids) delete g;
    cudaFree(sl->halo);
    cudaFree(sl->partials);
    cudaFree(sl->st);
    if (sl->st_host) cudaFreeHost(sl->st_host);
    delete sl;
}

}  // namespace

extern "C" {

int dare_slabs_create(dare_system* sys, int num_slabs, int num_levels, dare_slabs** out) {
    if (!sys || !out || num_levels < 1 || num_levels > 8) return DARE_ERR_BAD_ARG;
    *out = nullptr;
    dare_ctx* ctx = sys->grid->ctx;
    const GridDev& G = sys->grid->dev;
    if (num_slabs < 1 || num_slabs > kMaxSlabs)
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_slabs_create: 1 to 8 slabs");
    // every slab holds at least ng planes (the field exchange) and two (the operand halo)
    const int min_planes = G.ng > 2 ? G.ng : 2;
    if (G.n[0] / num_slabs < min_planes)
        return set_error(ctx, DARE_ERR_BAD_ARG, "dare_slabs_create: a slab needs at least num_ghost planes");
    cudaSetDevice(ctx->device);
    dare_slabs* sl = new (std::nothrow) dare_slabs();
    if (!sl) return DARE_ERR_OOM;
    sl->ctx = ctx;
    sl->device = ctx->device;
    sl->global = G;
    sl->ncomp = sys->ncomp;
    sl->S = num_slabs;
    sl->periodic_x = G.periodic[0];
    const int base = G.n[0] / num_slabs, extra = G.n[0] % num_slabs;
    int rc = DARE_OK;
    for (int s = 0; s < num_slabs && rc == DARE_OK; s++) {
        // planes [i0, i1): n0 split into runs, the first n0 % S one plane longer
        const int i0 = s * base + (s < extra ? s : extra);
        const int i1 = i0 + base + (s < extra ? 1 : 0);
        sl->i0.push_back(i0);
        sl->i1.push_back(i1);
        dare_grid* g = new (std::nothrow) dare_grid();
        if (!g) {
            rc = DARE_ERR_OOM;
            break;
        }
        g->ctx = ctx;
        g->dev = G;                      // the same cell widths, areas and volume, bit for bit
        g->dev.n[0] = i1 - i0;
        g->dev.gn[0] = (i1 - i0) + 2 * G.og[0];
        g->dev.periodic[0] = 0;          // the x neighbours are slabs (halo buffers), not a wrap
        g->dev.ncell = (int64_t)(i1 - i0) * G.n[1] * G.n[2];
        g->dev.ncell_ghosted = (int64_t)g->dev.gn[0] * G.gn[1] * G.gn[2];
        g->dev.origin[0] = G.origin[0] + i0 * G.dx[0];
        sl->grids.push_back(g);
        dare_field* f = nullptr;
        if ((rc = dare_field_create_n(g, num_levels, sys->ncomp, &f)) != DARE_OK) break;
        sl->fields.push_back(f);
        dare_system* sy = nullptr;
        if ((rc = dare_system_create_n(g, sys->ncomp, &sy)) != DARE_OK) break;
        sl->systems.push_back(sy);
        std::memcpy(sy->bc_type, sys->bc_type, sizeof(sy->bc_type));
        std::memcpy(sy->bc_value, sys->bc_value, sizeof(sy->bc_value));
        sy->bc_type_c = sys->bc_type_c;
        sy->bc_value_c = sys->bc_value_c;
        sy->xint = (lower(sl, s) >= 0 ? 1 : 0) | (upper(sl, s) >= 0 ? 2 : 0);
        if ((rc = ensure_solver_ws(sy)) != DARE_OK) break;
    }
    if (rc == DARE_OK) {
        const int budget = kMaxBlocks / num_slabs;
        for (int s = 0; s < num_slabs; s++) {
            MarchCfg m = march_config(ctx, sl->systems[s]->sdev, sizeof(double), budget);
            sl->item_base.push_back(sl->items_total);
            sl->items_total += m.nitems;
            sl->march.push_back(m);
            const int sb = grid_blocks(ctx, sl->systems[s]->sdev.ncell, 256, 8);
            sl->sblock_base.push_back(sl->sblocks_total);
            sl->sblocks_total += sb;
            sl->sblocks.push_back(sb);
        }
        if (sl->items_total > kMaxBlocks || sl->sblocks_total > kMaxBlocks)
            rc = set_error(ctx, DARE_ERR_UNSUPPORTED, "dare_slabs_create: too many work items for the reduction");
    }
    cudaError_t e = cudaSuccess;
    if (rc == DARE_OK) {
        e = cudaMalloc(&sl->halo, (size_t)num_slabs * 4 * sl->ncomp * plane_cells(sl) * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&sl->partials, (size_t)kMaxQ * kMaxBlocks * sizeof(double) + 64);
        if (e == cudaSuccess) e = cudaMalloc(&sl->st, sizeof(SolverState));
        if (e == cudaSuccess) e = cudaMemsetAsync(sl->st, 0, sizeof(SolverState), ctx->stream);
        if (e == cudaSuccess) e = cudaMallocHost(&sl->st_host, sizeof(SolverState));
        if (e != cudaSuccess) rc = check_cuda(ctx, e, "dare_slabs_create");
    }
    if (rc != DARE_OK) {
        slabs_free(sl);
        return rc == DARE_ERR_OOM ? set_error(ctx, rc, "dare_slabs_create: out of memory") : rc;
    }
    *out = sl;
    return DARE_OK;
}

int dare_slabs_destroy(dare_slabs* sl) {
    if (!sl) return DARE_ERR_BAD_ARG;
    cudaSetDevice(sl->device);
    slabs_free(sl);
    return DARE_OK;
}

int dare_slabs_count(const dare_slabs* sl) { return sl ? sl->S : DARE_ERR_BAD_ARG; }

int dare_slabs_range(const dare_slabs* sl, int slab, int64_t* i0, int64_t* i1) {
    if (!sl || slab < 0 || slab >= sl->S || !i0 || !i1) return DARE_ERR_BAD_ARG;
    *i0 = sl->i0[slab];
    *i1 = sl->i1[slab];
    return DARE_OK;
}

dare_system* dare_slabs_system(dare_slabs* sl, int slab) {
    return (sl && slab >= 0 && slab < sl->S) ? sl->systems[slab] : nullptr;
}

dare_field* dare_slabs_field(dare_slabs* sl, int slab) {
    return (sl && slab >= 0 && slab < sl->S) ? sl->fields[slab] : nullptr;
}

// dare_system_set_bc on every slab, checked against the whole grid
int dare_slabs_set_bc(dare_slabs* sl, int face, int type, double value) {
    if (!sl || face < DARE_WEST || face > DARE_TOP) return DARE_ERR_BAD_ARG;
    const int d = (face - 1) / 2;
    if (d >= sl->global.dim) return set_error(sl->ctx, DARE_ERR_BAD_ARG, "dare_slabs_set_bc: inactive dimension");
    if (sl->global.periodic[d] ? type != DARE_BC_PERIODIC : (type != DARE_BC_DIRICHLET && type != DARE_BC_NEUMANN))
        return set_error(sl->ctx, DARE_ERR_BAD_ARG, "dare_slabs_set_bc: condition does not fit the face");
    for (auto* sy : sl->systems) {
        sy->bc_type[face - 1] = type;
        sy->bc_value[face - 1] = value;
        for (int c = 0; c < (int)sy->bc_type_c.size() / 6; c++) {
            sy->bc_type_c[c * 6 + face - 1] = type;
            sy->bc_value_c[c * 6 + face - 1] = value;
        }
    }
    return DARE_OK;
}

// Every time level of the global field f into the slabs: each slab receives
// its planes with ng ghost planes on either side (the global field's own
// ghosts at a bounded end), as a rank receives its part of the initial field.
int dare_slabs_scatter(dare_slabs* sl, dare_field* f) {
    if (!sl || !f || f->ncomp != sl->ncomp || f->grid->dev.ncell_ghosted != sl->global.ncell_ghosted ||
        f->grid->dev.n[0] != sl->global.n[0] || f->num_levels < sl->fields[0]->num_levels)
        return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = sl->ctx;
    cudaSetDevice(ctx->device);
    const int64_t GP = ghosted_plane(sl);
    const size_t gcomp = (size_t)sl->global.ncell_ghosted * sizeof(double);   // one component of f
    int rc;
    for (int s = 0; s < sl->S; s++) {
        dare_field* sf = sl->fields[s];
        const size_t bytes = (size_t)sf->grid->dev.ncell_ghosted * sizeof(double);
        for (int l = 0; l < sf->num_levels; l++)
            if ((rc = transfer(ctx, sf->level[l], f->level[l] + (int64_t)sl->i0[s] * GP, bytes, sl->ncomp, bytes,
                               gcomp)))
                return rc;
    }
    return DARE_OK;
}

// The slabs' planes back into every level of the global field f (the first
// slab's lower and the last slab's upper ghost planes included).
int dare_slabs_gather(dare_slabs* sl, dare_field* f) {
    if (!sl || !f || f->ncomp != sl->ncomp || f->grid->dev.ncell_ghosted != sl->global.ncell_ghosted ||
        f->grid->dev.n[0] != sl->global.n[0] || f->num_levels < sl->fields[0]->num_levels)
        return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = sl->ctx;
    cudaSetDevice(ctx->device);
    const int64_t GP = ghosted_plane(sl);
    const int og = sl->global.og[0];
    const size_t gcomp = (size_t)sl->global.ncell_ghosted * sizeof(double);
    int rc;
    for (int s = 0; s < sl->S; s++) {
        dare_field* sf = sl->fields[s];
        const size_t scomp = (size_t)sf->grid->dev.ncell_ghosted * sizeof(double);
        const int ns = sl->i1[s] - sl->i0[s];
        const int p0 = s == 0 ? 0 : og;                            // first slab plane copied
        const int p1 = s == sl->S - 1 ? ns + 2 * og : og + ns;     // one past the last
        for (int l = 0; l < sf->num_levels; l++)
            if ((rc = transfer(ctx, f->level[l] + (int64_t)(sl->i0[s] + p0) * GP, sf->level[l] + (int64_t)p0 * GP,
                               (size_t)(p1 - p0) * GP * sizeof(double), sl->ncomp, gcomp, scomp)))
                return rc;
    }
    return DARE_OK;
}

// Field::ExchangeHaloCells on every slab: the periodic j / k ghosts inside
// the slab, then ng planes from each x neighbour into the ghost planes
// (whole ghosted planes, so their j / k ghosts travel too).
int dare_slabs_exchange_halo(dare_slabs* sl) {
    if (!sl) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = sl->ctx;
    cudaSetDevice(ctx->device);
    int rc;
    for (int s = 0; s < sl->S; s++)
        if ((rc = dare_field_exchange_halo(sl->fields[s]))) return rc;   // every component
    const int64_t GP = ghosted_plane(sl);
    const int og = sl->global.og[0];
    const size_t bytes = (size_t)og * GP * sizeof(double);
    auto comp = [&](int s) { return (size_t)sl->fields[s]->grid->dev.ncell_ghosted * sizeof(double); };
    for (int s = 0; s < sl->S; s++) {
        const int lo = lower(sl, s), hi = upper(sl, s);
        double* own = sl->fields[s]->level[0];
        const int ns = sl->i1[s] - sl->i0[s];
        if (lo >= 0) {
            const int nl = sl->i1[lo] - sl->i0[lo];
            if ((rc = transfer(ctx, own, sl->fields[lo]->level[0] + (int64_t)nl * GP, bytes, sl->ncomp, comp(s),
                               comp(lo))))
                return rc;
        }
        if (hi >= 0 && (rc = transfer(ctx, own + (int64_t)(og + ns) * GP, sl->fields[hi]->level[0] + (int64_t)og * GP,
                                      bytes, sl->ncomp, comp(s), comp(hi))))
            return rc;
    }
    return DARE_OK;
}

int dare_slabs_copy_to_old(dare_slabs* sl) {
    if (!sl) return DARE_ERR_BAD_ARG;
    for (auto* f : sl->fields) {
        const int rc = dare_field_copy_to_old(f);
        if (rc) return rc;
    }
    return DARE_OK;
}

// Trilinos::Build on every slab from its own field; descs[s] is slab s's
// descriptor (its face arrays cover its own planes: n_s + 1 x-faces, the
// last one the global face i1, face 0 on a periodic x for the last slab).
int dare_slabs_assemble(dare_slabs* sl, const dare_assembly_desc* descs) {
    if (!sl || !descs) return DARE_ERR_BAD_ARG;
    cudaSetDevice(sl->ctx->device);
    for (int s = 0; s < sl->S; s++) {
        dare_field* f = sl->fields[s];
        const double* phi_old = f->num_levels > 1 ? f->level[1] : f->level[0];
        const int rc = launch_assemble(sl->systems[s], &descs[s], f->level[0], phi_old);
        if (rc) return rc;
    }
    return DARE_OK;
}

// Trilinos::CopyTo on every slab
int dare_slabs_copy_to(dare_slabs* sl) {
    if (!sl) return DARE_ERR_BAD_ARG;
    for (int s = 0; s < sl->S; s++) {
        const int rc = dare_system_copy_to(sl->systems[s], sl->fields[s]);   // every component
        if (rc) return rc;
    }
    return DARE_OK;
}

// BiCGStab2 over all slabs' rows (FP64, plain or Jacobi), the steps of the
// single-grid solve with the operand planes exchanged before each SpMV and
// every reduction over all slabs.
int dare_slabs_solve(dare_slabs* sl, const dare_solver_params* p, dare_solve_report* rep) {
    if (!sl || !p || !rep) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = sl->ctx;
    if (p->max_it < 0 || !(p->tol >= 0.)) return set_error(ctx, DARE_ERR_BAD_ARG, "slab bicgstab2: bad params");
    if (p->precond != DARE_PREC_NONE && p->precond != DARE_PREC_JACOBI)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "slab bicgstab2: preconditioner not supported");
    if (p->precision != DARE_PRECISION_FP64)
        return set_error(ctx, DARE_ERR_UNSUPPORTED, "slab bicgstab2: FP64 only");
    cudaSetDevice(ctx->device);
    const bool jacobi = p->precond == DARE_PREC_JACOBI;
    const int S = sl->S;
    int rc;
    SolverState init{};
    init.tol = p->tol;
    init.max_it = p->max_it;
    init.tol_relative = p->tol_relative;
    DARE_CUDA(ctx, cudaMemcpyAsync(sl->st, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    if (jacobi) {   // invd on every slab, then Ahat = A D^-1 with the neighbours' invd planes
        std::vector<FFold> kf;
        for (int s = 0; s < S; s++) {
            dare_system* sy = sl->systems[s];
            const int64_t n = sy->sdev.ncell;
            k_invdiag<<<grid_blocks(ctx, n, 256, 8), 256, 0, ctx->stream>>>(sy->diag, sy->ws->invd, n);
            DARE_LAUNCHED(ctx);
            kf.push_back(make_fold(sy->diag, sy->ws->invd, sy->ws->ahat, n));
        }
        if ((rc = march_slabs(sl, kf))) return rc;
    }
    const SlabVecs v = slab_vectors(sl, jacobi);
    if (jacobi) {
        std::vector<FInit<double, true>> ki;
        for (int s = 0; s < S; s++) ki.push_back(make_init<double, true>(v.op[s], v.vs[s]));
        rc = march_slabs(sl, ki);
    } else {
        std::vector<FInit<double, false>> ki;
        for (int s = 0; s < S; s++) ki.push_back(make_init<double, false>(v.op[s], v.vs[s]));
        rc = march_slabs(sl, ki);
    }
    if (rc) return rc;
    rc = jacobi ? slab_run<true>(sl, v, p->max_it, p->check_every) : slab_run<false>(sl, v, p->max_it, p->check_every);
    if (rc) return rc;
    const SolverState st = *sl->st_host;
    for (int s = 0; s < S; s++)
        if ((rc = finish_step10(ctx, sl->systems[s]->sdev.ncell, st, sl->st, v.vs[s]))) return rc;
    std::memset(rep, 0, sizeof(*rep));
    rep->iters = st.k;
    rep->b_norm = sqrt(st.bnorm2);
    rep->res_abs = st.rnorm;
    rep->breakdown_step = st.step;
    rep->tol_abs = st.tol;
    if (st.status == ST_TAU0) {
        // BiCGStab2.inl:407-424, as in the single-grid solve
        if (jacobi && (rc = slab_scale(sl))) return rc;
        double tr = 0.;
        if ((rc = slab_true_residual(sl, &tr))) return rc;
        rep->res_abs = tr;
        if (tr <= st.tol) {
            rep->converged = 1;
            rep->status = DARE_SOLVE_CONVERGED;
            rep->breakdown_step = 0;
        } else {
            if (jacobi && (rc = slab_scale(sl))) return rc;
            rep->converged = 0;
            rep->status = DARE_SOLVE_BREAKDOWN;
        }
    } else {
        if (jacobi && (rc = slab_scale(sl))) return rc;
        rep->converged = st.rnorm <= st.tol;
        switch (st.status) {
        case ST_CONVERGED: rep->status = DARE_SOLVE_CONVERGED; break;
        case ST_MAXIT: rep->status = DARE_SOLVE_MAXIT; break;
        case ST_NAN: rep->status = DARE_SOLVE_NAN; break;
        default: rep->status = DARE_SOLVE_BREAKDOWN; break;
        }
    }
    if (p->compute_true_residual) {
        double tr = 0.;
        if ((rc = slab_true_residual(sl, &tr))) return rc;
        rep->true_res_abs = tr;
    }
    return DARE_OK;
}

// The reference's driver loop on every slab: Build, Solve, CopyTo,
// ExchangeHaloCells, CopyDataVectorsToOldTimeStep.
int dare_slabs_timestep(dare_slabs* sl, const dare_assembly_desc* descs, const dare_solver_params* p,
                        dare_solve_report* rep) {
    int rc = dare_slabs_assemble(sl, descs);
    if (rc) return rc;
    if ((rc = dare_slabs_solve(sl, p, rep))) return rc;
    if ((rc = dare_slabs_copy_to(sl))) return rc;
    if ((rc = dare_slabs_exchange_halo(sl))) return rc;
    return dare_slabs_copy_to_old(sl);
}

}  // extern "C"
