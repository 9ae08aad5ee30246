// The reference's own BiCGStab(2) (MatrixSystem/BiCGStab2.h, .inl), compiled
// from its header as it lies in the reference tree against the Belos /
// Teuchos / Kokkos stand-ins of oracle/ref_shim/, into
// oracle/_ref/libdare_ref.so.  Test infrastructure only: it checks the C
// restatement of the solve in dare_oracle.c.  Nothing in the product links or
// loads it.
//
// The vector and operator types below stand in for Tpetra's MultiVector and
// CrsMatrix (Trilinos 15), restating the definitions the solve relies on:
//   update(a, A, b):        this = a A + b this         (KokkosBlas axpby)
//   update(a, A, b, B, c):  this = a A + b B + c this   (KokkosBlas update)
//   dot / norm2:            OpenMP sums (in index order with one thread)
//   apply(x, y):            y_i = sum over the row's sorted columns of a_ip x_p
// and the right preconditioner is Ifpack2's RELAXATION Jacobi (one sweep,
// damping 1, zero start): y = D^-1 x with D^-1 = 1 / diag(A), as
// TrilinosSolver.inl:84-85,164-176 sets it up.  The loops are spread over the
// host threads as Tpetra's OpenMP node spreads them.
#include <cmath>
#include <cstdint>
#include <vector>

#include "Kokkos_Core.hpp"
#include "Tpetra_Map_decl.hpp"
#include "MatrixSystem/BiCGStab2.h"

namespace {

struct ShimMap {
    std::size_t n;
    Teuchos::RCP<const Teuchos::Comm<int>> comm;
    Teuchos::RCP<const Teuchos::Comm<int>> getComm() const { return comm; }
};

class ShimVector {
public:
    using map_type = ShimMap;
    using local_ordinal_type = int;
    using global_ordinal_type = long long;
    using node_type = Tpetra::HostNode;
    using scalar_type = double;
    using dot_type = double;

    ShimVector(const Teuchos::RCP<const map_type>& map, std::size_t /*num_vec*/) : map_(map), v(map->n, 0.) {}
    std::size_t getNumVectors() const { return 1; }
    Teuchos::RCP<const map_type> getMap() const { return map_; }
    void assign(const ShimVector& o) { v = o.v; }
    void putScalar(double a) {
        const int64_t n = (int64_t)v.size();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) v[i] = a;
    }
    void update(double a, const ShimVector& A, double b) {
        const int64_t n = (int64_t)v.size();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) v[i] = a * A.v[i] + b * v[i];
    }
    void update(double a, const ShimVector& A, double b, const ShimVector& B, double c) {
        const int64_t n = (int64_t)v.size();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) v[i] = a * A.v[i] + b * B.v[i] + c * v[i];
    }
    template <class View>
    void dot(const ShimVector& o, const View& out) const {
        const int64_t n = (int64_t)v.size();
        double s = 0.;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (int64_t i = 0; i < n; i++) s += v[i] * o.v[i];
        out[0] = s;
    }
    template <class View>
    void norm2(const View& out) const {
        const int64_t n = (int64_t)v.size();
        double s = 0.;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (int64_t i = 0; i < n; i++) s += v[i] * v[i];
        out[0] = std::sqrt(s);
    }

    std::vector<double> v;

private:
    Teuchos::RCP<const map_type> map_;
};

struct ShimCsr {
    int64_t n;
    const int64_t* rowptr;
    const int64_t* cols;
    const double* vals;
    void apply(const ShimVector& x, ShimVector& y) const {
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < n; r++) {
            double s = 0.;
            for (int64_t p = rowptr[r]; p < rowptr[r + 1]; p++) s += vals[p] * x.v[cols[p]];
            y.v[r] = s;
        }
    }
};

}  // namespace

extern "C" {
// Solves A x = b with the reference's BiCGStab2::solve (absolute-norm stop at
// tol, as its RNORM criterion fixes), Jacobi on the right when precond = 1.
// x holds the initial guess on entry and the solution on return.  Outputs the
// iteration count and whether it reports convergence.  Returns 0, or -1 when
// the solve throws.
int dref_bicgstab2(int64_t n, const int64_t* rowptr, const int64_t* cols, const double* vals, const double* b,
                   double* x, double tol, int max_it, int precond, int* iters, int* converged) {
    using Solver = dare::Matrix::BiCGStab2<double, ShimVector, ShimCsr>;
    auto map = Teuchos::rcp(new ShimMap{(std::size_t)n, Teuchos::rcp(new Teuchos::Comm<int>())});
    Teuchos::RCP<const ShimMap> cmap = map;
    auto X = Teuchos::rcp(new ShimVector(cmap, 1));
    auto B = Teuchos::rcp(new ShimVector(cmap, 1));
    for (int64_t i = 0; i < n; i++) {
        X->v[i] = x[i];
        B->v[i] = b[i];
    }
    auto A = Teuchos::rcp(new ShimCsr{n, rowptr, cols, vals});
    auto problem = Teuchos::rcp(new Belos::LinearProblem<double, ShimVector, ShimCsr>(A, X, B));
    std::vector<double> inv_diag;
    if (precond == 1) {
        inv_diag.assign(n, 0.);
        for (int64_t r = 0; r < n; r++) {
            double d = 0.;
            for (int64_t p = rowptr[r]; p < rowptr[r + 1]; p++)
                if (cols[p] == r) d = vals[p];
            inv_diag[r] = 1. / d;
        }
        problem->setRightPrec([&inv_diag](const ShimVector& in, ShimVector& out) {
            const int64_t m = (int64_t)in.v.size();
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < m; i++) out.v[i] = inv_diag[i] * in.v[i];
        });
    }
    auto params = Teuchos::rcp(new Teuchos::ParameterList());
    params->set("Convergence Tolerance", tol);
    params->set("Maximum Iterations", max_it);
    try {
        Solver solver(params);
        solver.setProblem(problem);
        const Belos::ReturnType ret = solver.solve();
        *iters = solver.getNumIters();
        *converged = ret == Belos::Converged;
    } catch (const std::exception&) {
        return -1;
    }
    for (int64_t i = 0; i < n; i++) x[i] = X->v[i];
    return 0;
}
}
