// The reference's own assembly path, compiled from its headers as they lie in
// the reference tree (Grid/Cartesian, Equations, Data, MatrixSystem) against
// the single-rank MPI / Kokkos / Tpetra stand-ins of oracle/ref_shim/, into
// oracle/_ref/libdare_ref.so.  Test infrastructure only: it checks the C
// restatement in dare_oracle.c against the code it restates.  Nothing in the
// product links or loads it.
//
// dref_assemble runs, per internal cell, exactly the loop of
// Trilinos<SC>::BuildNew (MatrixSystem/Trilinos.inl:285-385: Initialize,
// SetInitialGuess from the field, the user functor, Finalize, rows by global
// ordinal, columns sorted as fillComplete leaves them) with the functor the
// reference's drivers compose (test/Verification/counter_diffusion1D.cpp:
// 107-148, advection_periodic2D.cpp:108-126):
//     mb  = ddt(field);                          Equations/DDT.inl
//     mb += div(TVD(vel) * field);               Grid/Cartesian/TVD_Cartesian.inl:185-261
//     mb -= div(D, grad(mb));                    scalar D, Divergence_Cartesian.inl:90-96
//     mb -= div(Dface * grad(mb));               face D as a FaceValueStencil
//     fold the boundary faces W,E,S,N,B,T:       Dirichlet C -= X, rhs -= 2 bc X; Neumann C += X
// The TVD velocity is the constant-velocity constructor
// (TVD_Cartesian.inl:40-53), the one the reference's tests and drivers use.
// The header Grid/Cartesian/VTKOptions_Cartesian.h (VTK output options, not
// on this path) is kept out by defining its include guard on the command line.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "Grid/Cartesian.h"
#include "Data/Field.h"
#include "Equations/FluxLimiter.h"

extern "C" {
// Mirrors the fields of the oracle's dor_assembly that this path supports.
struct dref_desc {
    int dim;
    int64_t n[3];
    double L[3];
    int periodic[3];
    double dt;                 // > 0: DDT term
    int diffusion;             // 0 none, 1 scalar D, 2 face D arrays
    double D;
    const double* face_D[3];   // face arrays in the oracle's layout
    int convection;            // 0 none, 1 constant velocity
    double vel[3];
    int limiter;               // 0 CDS, 1 UPWIND, 2 VANALBADA, 3 MINMOD, 4 VANLEER
    int scheme;                // 0 EULER_BACKWARD, 1 EULER_FORWARD, 2 CRANK_NICHOLSON,
                               // 3 ADAMS_BASHFORT, 4 ADAMS_MOULTON
    int bc_type[6];            // faces W,E,S,N,B,T: 1 Dirichlet, 2 Neumann
    double bc_value[6];
    int ncomp;                 // 1 or 2 field components (0 reads as 1)
    int bc_type1[6];           // component 1's conditions (ncomp 2)
    double bc_value1[6];
};
}

namespace {

// van Leer, psi = (r + |r|) / (1 + |r|) with NaN -> 0, +inf -> 2, -inf -> 0:
// not in the reference; the same definition as the oracle and the GPU, in the
// interface of the reference's limiters (Equations/FluxLimiter.h).
struct VANLEER {
    template <std::size_t N, typename SC>
    static dare::utils::Vector<N, SC> GetValue(const dare::utils::Vector<N, SC>& r) {
        dare::utils::Vector<N, SC> ret;
        for (std::size_t n{0}; n < N; n++) ret[n] = GetValue(r[n]);
        return ret;
    }
    template <typename SC>
    static SC GetValue(SC r) {
        if (std::isnan(r)) return SC(0);
        if (std::isinf(r)) return r > 0 ? SC(2) : SC(0);
        const SC a = std::fabs(r);
        return (r + a) / (SC(1) + a);
    }
};

int64_t face_index(const dref_desc* d, int dd, int64_t i, int64_t j, int64_t k) {
    const int64_t n1 = d->dim > 1 ? d->n[1] : 1, n2 = d->dim > 2 ? d->n[2] : 1;
    switch (dd) {
    case 0: return (i * n1 + j) * n2 + k;
    case 1: return (i * (n1 + 1) + j) * n2 + k;
    default: return (i * n1 + j) * (n2 + 1) + k;
    }
}
int64_t upper_face(const dref_desc* d, int dd, int64_t i) {
    return (d->periodic[dd] && i + 1 == d->n[dd]) ? 0 : i + 1;
}

int grid_counter = 0;

template <std::size_t Dim, class Limiter, class Scheme, std::size_t N>
int assemble(const dref_desc* d, const double* phi_conv, const double* phi_old, int64_t* rowptr, int64_t* cols,
             double* vals, double* rhs, double* x0, int64_t nnz_cap) {
    using SC = double;
    using GO = dare::defaults::GlobalOrdinalType;
    using LO = dare::defaults::LocalOrdinalType;
    using Grid = dare::Grid::Cartesian<Dim>;
    using Field = dare::Data::Field<Grid, SC, N>;
    using CNB = typename Grid::NeighborID;
    using MB = dare::Matrix::MatrixBlock<Grid, GO, SC, N>;

    const int num_ghost = 2;
    dare::mpi::ExecutionManager exman(MPI_COMM_WORLD, dare::mpi::Verbosity::None);
    typename Grid::IndexGlobal res;
    typename Grid::VecSC size;
    typename Grid::Index periodic, staggered;
    for (std::size_t q = 0; q < Dim; q++) {
        res[q] = d->n[q];
        size[q] = d->L[q];
        periodic[q] = d->periodic[q];
        staggered[q] = 0;
    }
    Grid grid("dref_grid_" + std::to_string(grid_counter++), &exman, res, size, num_ghost, periodic);
    auto grep = grid.GetRepresentation(staggered);

    // ghosted field in the oracle's layout: extent n + 2 g along the grid's
    // dimensions, 1 along the others, last dimension fastest
    int64_t gn[3] = {1, 1, 1};
    for (std::size_t q = 0; q < Dim; q++) gn[q] = d->n[q] + 2 * num_ghost;
    // N components: the fields are given component after component, each in
    // the ghosted layout
    Field field("phi", grep, 2);
    const LO nloc = grep.GetNumberLocalCells();
    const int64_t gcells = gn[0] * gn[1] * gn[2];
    for (LO lo = 0; lo < nloc; lo++) {
        const auto ind = grep.MapOrdinalToIndexLocal(lo);
        int64_t idx[3] = {0, 0, 0};
        for (std::size_t q = 0; q < Dim; q++) idx[q] = ind[q];
        const int64_t off = (idx[0] * gn[1] + idx[1]) * gn[2] + idx[2];
        for (std::size_t n = 0; n < N; n++) {
            field.GetDataVector(0).At(lo, n) = phi_conv[n * gcells + off];
            field.GetDataVector(1).At(lo, n) = phi_old[n * gcells + off];
        }
    }

    typename Grid::VecSC velocity;
    for (std::size_t q = 0; q < Dim; q++) velocity[q] = d->vel[q];
    const int64_t nn[3] = {d->n[0], Dim > 1 ? d->n[1] : 1, Dim > 2 ? d->n[2] : 1};
    const CNB faces[6] = {CNB::WEST, CNB::EAST, CNB::SOUTH, CNB::NORTH, CNB::BOTTOM, CNB::TOP};

    auto functor = [&](MB* mb) {
        using Gradient = dare::Matrix::Gradient<Grid>;
        using Divergence = dare::Matrix::Divergence<Grid, Scheme>;
        using TVD = dare::Matrix::TVD<Grid, SC, Limiter>;
        using DDT = dare::Matrix::DDT<Grid>;
        auto g_r = mb->GetRepresentation();
        LO loc_o{mb->GetLocalOrdinal()};
        const GO glob = mb->GetGlobalOrdinal();
        const int64_t gi[3] = {glob / (nn[1] * nn[2]), (glob / nn[2]) % nn[1], glob % nn[2]};

        if (d->dt > 0.) {
            DDT ddt(*g_r, loc_o, d->dt);
            (*mb) = ddt(field);
        }
        if (d->convection == 1) {
            TVD tvd(*g_r, loc_o, velocity);
            Divergence div(*g_r, loc_o);
            (*mb) += div(tvd * field.GetDataVector());
        }
        if (d->diffusion == 1) {
            Gradient grad(*g_r, loc_o);
            Divergence div(*g_r, loc_o);
            (*mb) -= div(d->D, grad(*mb));
        } else if (d->diffusion == 2) {
            dare::Data::FaceValueStencil<Grid, SC, N> dface;   // the same face D for every component
            for (std::size_t q = 0; q < Dim; q++) {
                int64_t fi[3] = {gi[0], gi[1], gi[2]};
                const double lo = d->face_D[q][face_index(d, (int)q, fi[0], fi[1], fi[2])];
                fi[q] = upper_face(d, (int)q, fi[q]);
                const double up = d->face_D[q][face_index(d, (int)q, fi[0], fi[1], fi[2])];
                for (std::size_t n = 0; n < N; n++) {
                    dface.SetValue(faces[2 * q], n, lo);
                    dface.SetValue(faces[2 * q + 1], n, up);
                }
            }
            Gradient grad(*g_r, loc_o);
            Divergence div(*g_r, loc_o);
            (*mb) -= div(dface * grad(*mb));   // FaceValueStencil * FaceMatrixStencil, Stencils_Cartesian.inl:709-716
        }
        for (std::size_t q = 0; q < Dim; q++) {
            if (d->periodic[q]) continue;
            for (int side = 0; side < 2; side++) {
                const int f = 2 * (int)q + side;
                if (!(side == 0 ? gi[q] == 0 : gi[q] == nn[q] - 1)) continue;
                for (std::size_t n = 0; n < N; n++) {   // counter_diffusion1D.cpp:123-146, per component
                    const int type = n == 0 ? d->bc_type[f] : d->bc_type1[f];
                    const double value = n == 0 ? d->bc_value[f] : d->bc_value1[f];
                    const SC X = mb->Get(n, faces[f]);
                    if (type == 1) {
                        mb->Get(n, CNB::CENTER) -= X;
                        mb->GetRhs(n) -= 2. * value * X;
                    } else {
                        mb->Get(n, CNB::CENTER) += X;
                    }
                    mb->Remove(n, faces[f]);
                }
            }
        }
    };

    const LO ncell = grep.GetNumberLocalCellsInternal();
    std::vector<MB> blocks(ncell);
#pragma omp parallel for                        // as Trilinos.inl:308
    for (LO node = 0; node < ncell; node++) {   // Trilinos.inl:309-328
        MB* mb = &blocks[node];
        const GO node_global = grep.MapLocalToGlobalInternal(node);
        mb->Initialize(&grep, node_global);
        for (std::size_t n = 0; n < N; n++)
            mb->SetInitialGuess(n, field.GetDataVector().At(grep.MapInternalToLocal(node), n));
        functor(mb);
        mb->Finalize();
    }
    int64_t nnz = 0;
    rowptr[0] = 0;
    std::vector<std::pair<GO, SC>> row;
    for (LO node = 0; node < ncell; node++) {   // Trilinos.inl:370-384, rows in global order
        MB& mb = blocks[node];
        mb.Finalize();
        const GO r = grep.MapLocalToGlobalInternal(node);
        if (r != node) return -3;                // one rank: local and global internal ordinals agree
        for (std::size_t n = 0; n < N; n++) {    // row node * N + n (MatrixBlockBase::GetRow)
            const auto& c = mb.GetColumnOrdinals(n);
            const auto& v = mb.GetColumnValues(n);
            row.clear();
            for (std::size_t e = 0; e < c.size(); e++) row.emplace_back(c[e], v[e]);
            std::stable_sort(row.begin(), row.end(),
                             [](const std::pair<GO, SC>& a, const std::pair<GO, SC>& b) { return a.first < b.first; });
            for (std::size_t e = 0; e + 1 < row.size(); e++)
                if (row[e].first == row[e + 1].first) return -4;   // duplicate columns (a periodic extent < 3)
            if (nnz + (int64_t)row.size() > nnz_cap) return -2;
            for (const auto& cv : row) {
                cols[nnz] = cv.first;
                vals[nnz] = cv.second;
                nnz++;
            }
            const int64_t rr = (int64_t)node * N + n;
            rowptr[rr + 1] = nnz;
            rhs[rr] = mb.GetRhs(n);
            x0[rr] = mb.GetInitialGuess(n);
        }
    }
    return 0;
}

template <std::size_t Dim, class Limiter, class Scheme>
int by_ncomp(const dref_desc* d, const double* a, const double* b, int64_t* rp, int64_t* c, double* v, double* r,
             double* x, int64_t cap) {
    if (d->ncomp == 2) return assemble<Dim, Limiter, Scheme, 2>(d, a, b, rp, c, v, r, x, cap);
    if (d->ncomp <= 1) return assemble<Dim, Limiter, Scheme, 1>(d, a, b, rp, c, v, r, x, cap);
    return -1;
}

template <std::size_t Dim, class Limiter>
int by_scheme(const dref_desc* d, const double* a, const double* b, int64_t* rp, int64_t* c, double* v, double* r,
              double* x, int64_t cap) {
    switch (d->scheme) {
    case 0: return by_ncomp<Dim, Limiter, dare::Matrix::EULER_BACKWARD>(d, a, b, rp, c, v, r, x, cap);
    case 1: return by_ncomp<Dim, Limiter, dare::Matrix::EULER_FORWARD>(d, a, b, rp, c, v, r, x, cap);
    case 2: return by_ncomp<Dim, Limiter, dare::Matrix::CRANK_NICHOLSON>(d, a, b, rp, c, v, r, x, cap);
    case 3: return by_ncomp<Dim, Limiter, dare::Matrix::ADAMS_BASHFORT>(d, a, b, rp, c, v, r, x, cap);
    // ADAMS_MOULTON does not compile in the reference: its GetWeights is not
    // static (Equations/TimeDiscretizationSchemes.h:70), and Divergence calls
    // it as a static member (Divergence_Cartesian.inl:183).
    default: return -1;
    }
}

template <std::size_t Dim>
int by_limiter(const dref_desc* d, const double* a, const double* b, int64_t* rp, int64_t* c, double* v, double* r,
               double* x, int64_t cap) {
    switch (d->limiter) {
    case 0: return by_scheme<Dim, dare::Matrix::CDS>(d, a, b, rp, c, v, r, x, cap);
    case 1: return by_scheme<Dim, dare::Matrix::UPWIND>(d, a, b, rp, c, v, r, x, cap);
    case 2: return by_scheme<Dim, dare::Matrix::VANALBADA>(d, a, b, rp, c, v, r, x, cap);
    case 3: return by_scheme<Dim, dare::Matrix::MINMOD>(d, a, b, rp, c, v, r, x, cap);
    case 4: return by_scheme<Dim, VANLEER>(d, a, b, rp, c, v, r, x, cap);
    default: return -1;
    }
}

}  // namespace

extern "C" {
// Assembles the system of one implicit step with the reference's own
// operators.  phi_conv / phi_old: ghosted fields (two ghost layers) in the
// oracle's layout, component after component.  Outputs: CSR rows (rowptr
// rows+1, cols / vals up to nnz_cap),
// rhs and initial guess per row (cell * ncomp + component).  Returns 0, or -1 (bad
// description, or a scheme the reference does not compile), -2 (nnz_cap too
// small), -3 / -4 (unsupported layout).
int dref_assemble(const dref_desc* d, const double* phi_conv, const double* phi_old, int64_t* rowptr, int64_t* cols,
                  double* vals, double* rhs, double* x0, int64_t nnz_cap) {
    if (d->convection && d->convection != 1) return -1;
    switch (d->dim) {
    case 1: return by_limiter<1>(d, phi_conv, phi_old, rowptr, cols, vals, rhs, x0, nnz_cap);
    case 2: return by_limiter<2>(d, phi_conv, phi_old, rowptr, cols, vals, rhs, x0, nnz_cap);
    case 3: return by_limiter<3>(d, phi_conv, phi_old, rowptr, cols, vals, rhs, x0, nnz_cap);
    default: return -1;
    }
}
}
