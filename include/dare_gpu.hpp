// dare_gpu.hpp -- C++ host API over the C ABI of dare_gpu.h.
//
// Mirrors the host-side types of hpc-dave/dare's finite-volume path so a
// DaRe time loop maps one to one onto device calls:
//
//   dare::Grid::Cartesian<Dim>          -> dare_b200::Cartesian      (CartesianMesh.h:177-379)
//   dare::Data::Field<Grid,SC,1>        -> dare_b200::Field          (Data/Field.h:47-138)
//   dare::Matrix::Trilinos<SC>          -> dare_b200::Trilinos       (MatrixSystem/Trilinos.h:51-314)
//   dare::Matrix::MatrixBlock (functor) -> dare_b200::Assembly       (the fused per-cell functor),
//                                          dare_b200::MatrixBlock    (a composed functor: ddt, div(grad),
//                                                                     div(TVD * field) terms with =, +=, -=, Add)
//                                          or Trilinos::SetBlocks    (host-built coefficients)
//   dare::Matrix::BiCGStab2 / TrilinosSolver::Solve("BICGSTAB2")
//                                       -> dare_b200::BiCGStab2      (BiCGStab2.h:58-206)
//
// Errors become dare_b200::Error exceptions (the C ABI itself never throws
// or aborts).  Objects own their handles (RAII, move-only).
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dare_gpu.h"

namespace dare_b200 {

class Error : public std::runtime_error {
public:
    Error(const std::string& what, int code) : std::runtime_error(what), code(code) {}
    int code;
};

inline void check(int rc, dare_ctx* ctx, const char* what) {
    if (rc != DARE_OK) {
        std::string msg = std::string(what) + " failed (" + std::to_string(rc) + ")";
        if (ctx) msg += ": " + std::string(dare_ctx_last_error(ctx));
        throw Error(msg, rc);
    }
}

// One device and one CUDA stream.
class Context {
public:
    explicit Context(int device = 0) { check(dare_ctx_create(device, &h_), nullptr, "dare_ctx_create"); }
    ~Context() {
        if (h_) dare_ctx_destroy(h_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    dare_ctx* get() const { return h_; }
    void Synchronize() const { check(dare_ctx_synchronize(h_), h_, "synchronize"); }
    void SetStream(void* cuda_stream) { check(dare_ctx_set_stream(h_, cuda_stream), h_, "set_stream"); }

private:
    dare_ctx* h_ = nullptr;
};

// Grid::Cartesian<Dim> with its representation (np = 1, not staggered).
class Cartesian {
public:
    // staggered: the representation grid->GetRepresentation(Options(staggered...))
    // (CartesianRepresentation.inl:33-76); empty for the cell-centred one
    Cartesian(Context& ctx, std::vector<int64_t> resolution, std::vector<double> size, int num_ghost = 2,
              std::vector<int> periodic = {}, std::vector<int> staggered = {})
        : ctx_(&ctx) {
        const int dim = (int)resolution.size();
        int64_t n[3] = {1, 1, 1};
        double s[3] = {1., 1., 1.};
        int p[3] = {0, 0, 0}, st[3] = {0, 0, 0};
        for (int d = 0; d < dim && d < 3; d++) {
            n[d] = resolution[d];
            s[d] = d < (int)size.size() ? size[d] : 1.;
            p[d] = d < (int)periodic.size() ? periodic[d] : 0;
            st[d] = d < (int)staggered.size() ? staggered[d] : 0;
        }
        check(dare_grid_create_staggered(ctx.get(), dim, n, s, num_ghost, p, st, &h_), ctx.get(), "dare_grid_create");
        check(dare_grid_get_info(h_, &info_), ctx.get(), "dare_grid_get_info");
    }
    ~Cartesian() {
        if (h_) dare_grid_destroy(h_);
    }
    Cartesian(const Cartesian&) = delete;
    Cartesian& operator=(const Cartesian&) = delete;

    dare_grid* get() const { return h_; }
    Context& GetContext() const { return *ctx_; }
    const dare_grid_info& Info() const { return info_; }
    int64_t GetNumberLocalCellsInternal() const { return info_.num_cells; }
    int64_t GetNumberLocalCells() const { return info_.num_cells_ghosted; }
    double GetCellVolume() const { return info_.volume; }
    std::array<double, 3> GetDistances() const { return {info_.dx[0], info_.dx[1], info_.dx[2]}; }
    std::array<double, 3> GetFaceArea() const { return {info_.area[0], info_.area[1], info_.area[2]}; }
    // MapIndexToOrdinalLocalInternal (CartesianRepresentation.inl:371-384)
    int64_t MapIndexToOrdinalInternal(int64_t i, int64_t j = 0, int64_t k = 0) const {
        return (i * info_.n[1] + j) * info_.n[2] + k;
    }
    // Ghosted ("local") ordinal of an internal index
    int64_t MapInternalToLocal(int64_t i, int64_t j = 0, int64_t k = 0) const {
        const int g = info_.num_ghost;
        const int64_t gi = i + g, gj = info_.dim > 1 ? j + g : j, gk = info_.dim > 2 ? k + g : k;
        return (gi * info_.n_ghosted[1] + gj) * info_.n_ghosted[2] + gk;
    }

private:
    Context* ctx_;
    dare_grid* h_ = nullptr;
    dare_grid_info info_{};
};

// Field: time levels of ghosted GridVectors on the device (level 0 = new).
class Field {
public:
    // num_components: Field<Grid,SC,N>; host arrays interleave them (cell * N + c)
    Field(Cartesian& grid, int num_timesteps = 2, int num_components = 1) : grid_(&grid) {
        check(dare_field_create_n(grid.get(), num_timesteps, num_components, &h_), ctx(), "dare_field_create");
    }
    ~Field() {
        if (h_) dare_field_destroy(h_);
    }
    Field(const Field&) = delete;
    Field& operator=(const Field&) = delete;
    dare_field* get() const { return h_; }
    Cartesian& GetGrid() const { return *grid_; }

    int GetNumComponents() const { return dare_field_num_components(h_); }
    void Upload(const std::vector<double>& ghosted, int level = 0) {
        if ((int64_t)ghosted.size() != grid_->GetNumberLocalCells() * GetNumComponents())
            throw Error("Field::Upload: size", DARE_ERR_BAD_ARG);
        check(dare_field_upload(h_, level, ghosted.data()), ctx(), "dare_field_upload");
    }
    std::vector<double> Download(int level = 0) const {
        std::vector<double> v((size_t)(grid_->GetNumberLocalCells() * GetNumComponents()));
        check(dare_field_download(h_, level, v.data()), ctx(), "dare_field_download");
        return v;
    }
    void SetValues(double value, int level = 0) {
        Upload(std::vector<double>((size_t)(grid_->GetNumberLocalCells() * GetNumComponents()), value), level);
    }
    // Field::ExchangeHaloCells (Field.inl:100-103)
    void ExchangeHaloCells() { check(dare_field_exchange_halo(h_), ctx(), "exchange_halo"); }
    // Field::CopyDataVectorsToOldTimeStep (Field.inl:88-93)
    void CopyDataVectorsToOldTimeStep() { check(dare_field_copy_to_old(h_), ctx(), "copy_to_old"); }

private:
    dare_ctx* ctx() const { return grid_->GetContext().get(); }
    Cartesian* grid_;
    dare_field* h_ = nullptr;
};

enum class Limiter { CDS = DARE_LIMITER_CDS, UPWIND = DARE_LIMITER_UPWIND, VANALBADA = DARE_LIMITER_VANALBADA,
                     MINMOD = DARE_LIMITER_MINMOD, VANLEER = DARE_LIMITER_VANLEER };

// Time discretisation of the div(...) terms (Equations/TimeDiscretizationSchemes.h).
enum class TimeScheme : int {
    EULER_BACKWARD = DARE_SCHEME_EULER_BACKWARD,
    EULER_FORWARD = DARE_SCHEME_EULER_FORWARD,
    CRANK_NICHOLSON = DARE_SCHEME_CRANK_NICHOLSON,
    ADAMS_BASHFORTH = DARE_SCHEME_ADAMS_BASHFORTH,
    ADAMS_MOULTON = DARE_SCHEME_ADAMS_MOULTON
};

// The fused per-cell functor: mb = ddt(field); mb += div(TVD(vel) * field);
// mb -= div(D, grad(mb)); then the boundary folding of Trilinos::SetBC.
struct Assembly {
    double dt = 0.;
    double D = 0.;
    bool diffusion = false;
    const double* face_D[3] = {nullptr, nullptr, nullptr};     // device face arrays (optional)
    bool convection = false;
    std::array<double, 3> velocity{0., 0., 0.};
    const double* face_velocity[3] = {nullptr, nullptr, nullptr};  // device face arrays (optional)
    Limiter limiter = Limiter::VANLEER;
    TimeScheme scheme = TimeScheme::EULER_BACKWARD;

    dare_assembly_desc Desc() const {
        dare_assembly_desc d{};
        d.dt = dt;
        d.diffusion = face_D[0] ? 2 : (diffusion ? 1 : 0);
        d.D = D;
        d.convection = face_velocity[0] ? 2 : (convection ? 1 : 0);
        d.limiter = (int)limiter;
        d.scheme = (int)scheme;
        for (int i = 0; i < 3; i++) {
            d.face_D[i] = face_D[i];
            d.face_vel[i] = face_velocity[i];
            d.vel[i] = velocity[i];
        }
        return d;
    }
};

// One operator of a composed functor (Equations/Operators.h: DDT,
// Divergence of Gradient, Divergence of TVD * field), to be placed into a
// MatrixBlock with =, +=, -= or Add(component, ...).
struct Term {
    dare_term t{};
};
// ddt(field): implicit Euler with step dt (DDT.inl:39-81)
inline Term DDT(double dt) {
    Term r;
    r.t.kind = DARE_TERM_DDT;
    r.t.dt = dt;
    return r;
}
// Any other expression, evaluated by the caller on the device: per-cell
// values of the 7 slots (CENTER .. TOP; null: 0) and of the right-hand side
inline Term Coefficients(const double* const coef[7], const double* rhs) {
    Term r;
    r.t.kind = DARE_TERM_COEFFS;
    for (int q = 0; q < 7; q++) r.t.coef[q] = coef ? coef[q] : nullptr;
    r.t.coef_rhs = rhs;
    return r;
}
// div(D, grad(mb)) (D = 1: div(grad(mb))), or with device face diffusivities
inline Term DivGrad(double D = 1., TimeScheme scheme = TimeScheme::EULER_BACKWARD) {
    Term r;
    r.t.kind = DARE_TERM_DIFFUSION;
    r.t.D = D;
    r.t.scheme = (int)scheme;
    return r;
}
inline Term DivGrad(const double* const face_D[3], TimeScheme scheme = TimeScheme::EULER_BACKWARD) {
    Term r = DivGrad(1., scheme);
    for (int d = 0; d < 3; d++) r.t.face_D[d] = face_D[d];
    return r;
}
// div(TVD(u) * field) with a constant velocity or device face velocities
inline Term DivTVD(const std::array<double, 3>& u, Limiter limiter = Limiter::VANLEER,
                   TimeScheme scheme = TimeScheme::EULER_BACKWARD) {
    Term r;
    r.t.kind = DARE_TERM_CONVECTION;
    for (int d = 0; d < 3; d++) r.t.vel[d] = u[d];
    r.t.limiter = (int)limiter;
    r.t.scheme = (int)scheme;
    return r;
}
inline Term DivTVD(const double* const face_velocity[3], Limiter limiter = Limiter::VANLEER,
                   TimeScheme scheme = TimeScheme::EULER_BACKWARD) {
    Term r = DivTVD(std::array<double, 3>{0., 0., 0.}, limiter, scheme);
    for (int d = 0; d < 3; d++) r.t.face_vel[d] = face_velocity[d];
    return r;
}

// A composed per-cell functor written the way a DaRe functor writes its
// MatrixBlock (MatrixBlock_Cartesian.inl:480-593):
//     MatrixBlock mb;
//     mb = DDT(dt);                           // (*mblock) = ddt(field)
//     mb -= DivGrad();                        // (*mblock) -= div(grad(*mblock))
//     mb.Add(0, DivTVD({1., 0., 0.}));        // mblock->Add(0, div(u_0 * field).GetSlice(0))
//     system.Build(field, mb);
// The device evaluates the terms in order for every cell (dare_assemble_terms);
// per-component boundary folding comes from Trilinos::SetBC.
class MatrixBlock {
public:
    MatrixBlock& operator=(const Term& term) { return push(term, DARE_OP_SET, -1); }
    MatrixBlock& operator+=(const Term& term) { return push(term, DARE_OP_ADD, -1); }
    MatrixBlock& operator-=(const Term& term) { return push(term, DARE_OP_SUB, -1); }
    MatrixBlock& Set(int component, const Term& term) { return push(term, DARE_OP_SET, component); }
    MatrixBlock& Add(int component, const Term& term) { return push(term, DARE_OP_ADD, component); }
    MatrixBlock& Subtract(int component, const Term& term) { return push(term, DARE_OP_SUB, component); }
    const std::vector<dare_term>& Terms() const { return terms_; }
    void Clear() { terms_.clear(); }

private:
    MatrixBlock& push(const Term& term, int op, int component) {
        dare_term t = term.t;
        t.op = op;
        t.component = component;
        terms_.push_back(t);
        return *this;
    }
    std::vector<dare_term> terms_;
};

// Matrix::Trilinos<SC>: A, x, B of the structured system on the device.
class Trilinos {
public:
    // num_components: one 7-point stencil per component, rows cell * N + c
    explicit Trilinos(Cartesian& grid, int num_components = 1) : grid_(&grid) {
        check(dare_system_create_n(grid.get(), num_components, &h_), ctx(), "dare_system_create");
    }
    ~Trilinos() {
        if (h_) dare_system_destroy(h_);
    }
    Trilinos(const Trilinos&) = delete;
    Trilinos& operator=(const Trilinos&) = delete;
    dare_system* get() const { return h_; }

    // Dirichlet / Neumann folding of a non-periodic face (DARE_WEST..DARE_TOP),
    // for every component or for one
    void SetBC(int face, int type, double value = 0., int component = -1) {
        check(dare_system_set_bc_component(h_, component, face, type, value), ctx(), "dare_system_set_bc");
    }
    // Trilinos<SC>::Build(grep, field, functor, rebuild) with the fused functor
    // (Trilinos.inl:48-60).  `rebuild` picks the reference's BuildReplace
    // (keep the matrix graph, replace values) over BuildNew.  The device keeps
    // one fixed 7-slot structure per grid and rewrites it on every build, so
    // both give the same system whenever the functor's pattern is the same as
    // in the previous build, as in every driver loop of the reference.  (For a
    // functor that changes its pattern between builds, the reference's
    // BuildReplace keeps the previous values of entries the new build removes
    // -- Tpetra replaceLocalValues only touches the columns it is given; here
    // the new pattern is taken.)
    void Build(Field& field, const Assembly& functor, bool rebuild = false) {
        (void)rebuild;
        dare_assembly_desc d = functor.Desc();
        check(dare_assemble(h_, &d, field.get()), ctx(), "dare_assemble");
    }
    // ... and with a composed functor
    void Build(Field& field, const MatrixBlock& functor, bool rebuild = false) {
        (void)rebuild;
        const auto& t = functor.Terms();
        check(dare_assemble_terms(h_, t.data(), (int)t.size(), field.get()), ctx(), "dare_assemble_terms");
    }
    // Host-built MatrixBlocks: SoA diag[7][cells * N] (slots CENTER..TOP, rows
    // cell * N + c), rhs, x0
    void SetBlocks(const std::vector<double>& diag7, const std::vector<double>& rhs, const std::vector<double>& x0) {
        check(dare_system_set_coefficients(h_, diag7.data(), rhs.data(), x0.data()), ctx(), "set_coefficients");
    }
    int GetNumComponents() const { return dare_system_num_components(h_); }
    Cartesian& GetGrid() const { return *grid_; }
    std::vector<double> GetX() const {
        std::vector<double> x((size_t)(grid_->GetNumberLocalCellsInternal() * GetNumComponents()));
        check(dare_system_get_solution(h_, x.data()), ctx(), "get_solution");
        return x;
    }
    // Trilinos::CopyTo (Trilinos.inl:166-177)
    void CopyTo(Field& field) { check(dare_system_copy_to(h_, field.get()), ctx(), "copy_to"); }
    // CSR rows sorted by column, as Trilinos::PrintRow shows them
    void ExportCSR(std::vector<int64_t>& rowptr, std::vector<int64_t>& cols, std::vector<double>& vals) {
        const int64_t nnz = dare_system_csr_nnz(h_);
        rowptr.resize((size_t)(grid_->GetNumberLocalCellsInternal() * GetNumComponents()) + 1);
        cols.resize((size_t)nnz);
        vals.resize((size_t)nnz);
        check(dare_system_export_csr(h_, rowptr.data(), cols.data(), vals.data()), ctx(), "export_csr");
    }

private:
    dare_ctx* ctx() const { return grid_->GetContext().get(); }
    Cartesian* grid_;
    dare_system* h_ = nullptr;
};

// Matrix::BiCGStab2 with its Teuchos parameter names.
class BiCGStab2 {
public:
    enum class ReturnType { Converged, Unconverged };

    explicit BiCGStab2(const std::map<std::string, double>& params = {}) {
        dare_solver_params_default(&p_);
        auto it = params.find("Convergence Tolerance");
        if (it != params.end()) p_.tol = it->second;
        it = params.find("Maximum Iterations");
        if (it != params.end()) p_.max_it = (int)it->second;
    }
    dare_solver_params& Params() { return p_; }
    void SetPreconditioner(int precond) { p_.precond = precond; }
    void SetRelativeTolerance(bool rel) { p_.tol_relative = rel ? 1 : 0; }
    void SetMixedPrecision(bool on) { p_.precision = on ? DARE_PRECISION_FP32_REFINE : DARE_PRECISION_FP64; }

    ReturnType Solve(Trilinos& sys) {
        check(dare_bicgstab2_solve(sys.get(), &p_, &rep_), nullptr, "dare_bicgstab2_solve");
        return rep_.converged ? ReturnType::Converged : ReturnType::Unconverged;
    }
    // One step of the driver loop: Build, Solve, CopyTo, ExchangeHaloCells, CopyDataVectorsToOldTimeStep
    ReturnType TimeStep(Trilinos& sys, Field& field, const Assembly& functor) {
        dare_assembly_desc d = functor.Desc();
        check(dare_timestep(sys.get(), field.get(), &d, &p_, &rep_), nullptr, "dare_timestep");
        return rep_.converged ? ReturnType::Converged : ReturnType::Unconverged;
    }
    // ... with a composed functor
    ReturnType TimeStep(Trilinos& sys, Field& field, const MatrixBlock& functor) {
        sys.Build(field, functor);
        const ReturnType r = Solve(sys);
        sys.CopyTo(field);
        field.ExchangeHaloCells();
        field.CopyDataVectorsToOldTimeStep();
        return r;
    }
    int getNumIters() const { return rep_.iters; }
    double achievedTol() const { return rep_.res_abs; }
    const dare_solve_report& Report() const { return rep_; }

private:
    dare_solver_params p_{};
    dare_solve_report rep_{};
};

// The grid of a system distributed over slabs of i-planes, as the reference
// distributes it over ranks (CartesianDistribution.h:94-380), all slabs on
// the system's device: per slab its own field, rows and solver vectors.
class Slabs {
public:
    Slabs(Trilinos& sys, int num_slabs, int num_levels = 2) : ctx_(sys.GetGrid().GetContext().get()) {
        check(dare_slabs_create(sys.get(), num_slabs, num_levels, &h_), ctx_, "dare_slabs_create");
    }
    ~Slabs() {
        if (h_) dare_slabs_destroy(h_);
    }
    Slabs(const Slabs&) = delete;
    Slabs& operator=(const Slabs&) = delete;
    dare_slabs* get() const { return h_; }
    int Count() const { return dare_slabs_count(h_); }
    // planes [i0, i1) of slab s
    std::array<int64_t, 2> Range(int s) const {
        std::array<int64_t, 2> r{};
        check(dare_slabs_range(h_, s, &r[0], &r[1]), ctx_, "dare_slabs_range");
        return r;
    }
    void Scatter(Field& field) { check(dare_slabs_scatter(h_, field.get()), ctx_, "dare_slabs_scatter"); }
    void Gather(Field& field) { check(dare_slabs_gather(h_, field.get()), ctx_, "dare_slabs_gather"); }
    void ExchangeHaloCells() { check(dare_slabs_exchange_halo(h_), ctx_, "dare_slabs_exchange_halo"); }
    // Trilinos::Build on every slab, descs[s] holding slab s's face arrays
    void Build(const std::vector<Assembly>& functors) {
        const std::vector<dare_assembly_desc> d = Descs(functors);
        check(dare_slabs_assemble(h_, d.data()), ctx_, "dare_slabs_assemble");
    }
    BiCGStab2::ReturnType Solve(BiCGStab2& solver, dare_solve_report* rep = nullptr) {
        dare_solve_report r{};
        check(dare_slabs_solve(h_, &solver.Params(), &r), ctx_, "dare_slabs_solve");
        if (rep) *rep = r;
        return r.converged ? BiCGStab2::ReturnType::Converged : BiCGStab2::ReturnType::Unconverged;
    }
    // Build, Solve, CopyTo, ExchangeHaloCells, CopyDataVectorsToOldTimeStep on every slab
    BiCGStab2::ReturnType TimeStep(BiCGStab2& solver, const std::vector<Assembly>& functors,
                                   dare_solve_report* rep = nullptr) {
        const std::vector<dare_assembly_desc> d = Descs(functors);
        dare_solve_report r{};
        check(dare_slabs_timestep(h_, d.data(), &solver.Params(), &r), ctx_, "dare_slabs_timestep");
        if (rep) *rep = r;
        return r.converged ? BiCGStab2::ReturnType::Converged : BiCGStab2::ReturnType::Unconverged;
    }

private:
    std::vector<dare_assembly_desc> Descs(const std::vector<Assembly>& functors) const {
        if ((int)functors.size() != Count()) throw Error("Slabs: one functor per slab", DARE_ERR_BAD_ARG);
        std::vector<dare_assembly_desc> d;
        for (const auto& f : functors) d.push_back(f.Desc());
        return d;
    }
    dare_ctx* ctx_;
    dare_slabs* h_ = nullptr;
};

}  // namespace dare_b200
