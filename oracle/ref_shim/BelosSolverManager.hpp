// Belos::SolverManager, LinearProblem and the enums the reference's BiCGStab2
// (MatrixSystem/BiCGStab2.h, .inl) derives from and names, for the parity
// checker (oracle/_ref).  Test infrastructure only.  LinearProblem keeps the
// operator, the vectors and an optional right preconditioner given as a
// function y = M x, which is all BiCGStab2::solve asks of it.
#pragma once

#include <functional>
#include <string>

#include "Teuchos_shim.hpp"

namespace Belos {
enum ReturnType { Converged, Unconverged };
enum ResetType { Problem = 0x1, RecycleSubspace = 0x2 };

template <class SC, class MV, class OP>
class StatusTest {};

template <class SC, class MV, class OP>
class StatusTestCombo {
public:
    enum ComboType { AND, OR, SEQ };
};

template <class SC, class MV, class OP>
class LinearProblem {
public:
    using Prec = std::function<void(const MV&, MV&)>;
    LinearProblem(const Teuchos::RCP<const OP>& A, const Teuchos::RCP<MV>& X, const Teuchos::RCP<const MV>& B)
        : A_(A), X_(X), B_(B) {}
    void setRightPrec(Prec m) { right_ = std::move(m); }
    bool isLeftPrec() const { return false; }
    bool isRightPrec() const { return static_cast<bool>(right_); }
    void applyRightPrec(const MV& x, MV& y) const {
        if (right_)
            right_(x, y);
        else
            y.assign(x);
    }
    void applyLeftPrec(const MV& x, MV& y) const { y.assign(x); }
    Teuchos::RCP<MV> getLHS() const { return X_; }
    Teuchos::RCP<const MV> getRHS() const { return B_; }
    Teuchos::RCP<const OP> getOperator() const { return A_; }

private:
    Teuchos::RCP<const OP> A_;
    Teuchos::RCP<MV> X_;
    Teuchos::RCP<const MV> B_;
    Prec right_;
};

template <class SC, class MV, class OP>
class SolverManager {
public:
    virtual ~SolverManager() = default;
    virtual Teuchos::RCP<SolverManager<SC, MV, OP>> clone() const = 0;
    virtual const LinearProblem<SC, MV, OP>& getProblem() const = 0;
    virtual Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const = 0;
    virtual Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const = 0;
    virtual int getNumIters() const = 0;
    virtual bool isLOADetected() const = 0;
    virtual void setProblem(const Teuchos::RCP<LinearProblem<SC, MV, OP>>& problem) = 0;
    virtual void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) = 0;
    virtual void reset(const ResetType type) = 0;
    virtual ReturnType solve() = 0;
    virtual std::string description() const { return "Belos::SolverManager"; }
};
}  // namespace Belos
