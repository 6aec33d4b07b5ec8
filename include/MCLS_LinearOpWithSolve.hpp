// MCLS_LinearOpWithSolve.hpp -- the Stratimikos-facing solver: a linear
// operator with solves over blocks of right-hand sides, and its factory.
//
// The reference reaches Thyra/Stratimikos users through
// Thyra::MCLSLinearOpWithSolveFactory ("Solver Type", "Solver Types",
// "Convergence Test Frequency";
// thyra/src/Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:58-615),
// Thyra::MCLSLinearOpWithSolve
// (thyra/src/Thyra_MCLSLinearOpWithSolve_impl.hpp:52-430),
// MCLS::SolverManagerAdapter (thyra/src/MCLS_SolverManagerAdapter_impl.hpp:56-160)
// and MCLS::LinearProblemAdapter (thyra/src/MCLS_LinearProblemAdapter.hpp:100-270).
// Its factory creates AdjointSolverManager and ForwardSolverManager
// (Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:499-531), classes the library
// no longer has, so that code does not compile.  This header holds the same
// machinery without Thyra types:
//
// * the solve vocabulary (EOpTransp, SolveMeasureType, SolveCriteria,
//   SolveStatus) keeps Thyra's names and meaning;
// * a block of vectors is reached through MultiVectorTraits (HostMultiVector
//   is a ready-made host block);
// * "Solver Type" maps onto the managers of this library, so every solve runs
//   on the GPU: "MCSA" -> "Adjoint MCSA", "Adjoint MC", "Forward MC",
//   "Fixed Point", "Anderson" -> "Adjoint Anderson", and the SolverFactory
//   names "Adjoint MCSA", "Forward MCSA", "Adjoint Anderson" and
//   "Forward Anderson" as well.
//
// A Thyra::LinearOpWithSolveFactoryBase subclass that forwards to
// LinearOpWithSolveFactory (extracting the Tpetra matrix and multi-vectors
// from the Thyra wrappers) needs Trilinos and is not part of this header.
#ifndef MCLS_LINEAROPWITHSOLVE_HPP
#define MCLS_LINEAROPWITHSOLVE_HPP

#include <chrono>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "MCLS_PreconditionerFactory.hpp"
#include "MCLS_SolverFactory.hpp"

namespace MCLS {

// ---------------------------------------------------------------------------
// Solve vocabulary (Thyra_OperatorVectorTypes.hpp, Thyra_SolveSupportTypes.hpp)
// ---------------------------------------------------------------------------

enum EOpTransp { NOTRANS, CONJ, TRANS, CONJTRANS };

enum ESupportSolveUse {
    SUPPORT_SOLVE_UNSPECIFIED,
    SUPPORT_SOLVE_FORWARD_ONLY,
    SUPPORT_SOLVE_TRANSPOSE_ONLY,
    SUPPORT_SOLVE_FORWARD_AND_TRANSPOSE
};

enum EPreconditionerInputType {
    PRECONDITIONER_INPUT_TYPE_AS_OPERATOR,
    PRECONDITIONER_INPUT_TYPE_AS_MATRIX
};

enum ESolveMeasureNormType {
    SOLVE_MEASURE_ONE,
    SOLVE_MEASURE_NORM_RESIDUAL,
    SOLVE_MEASURE_NORM_SOLUTION,
    SOLVE_MEASURE_NORM_INIT_RESIDUAL,
    SOLVE_MEASURE_NORM_RHS
};

// The quantity numerator / denominator a requested tolerance bounds; ONE /
// ONE asks for the solver's own convergence test.
struct SolveMeasureType {
    ESolveMeasureNormType numerator = SOLVE_MEASURE_ONE;
    ESolveMeasureNormType denominator = SOLVE_MEASURE_ONE;
    SolveMeasureType() = default;
    SolveMeasureType(ESolveMeasureNormType n, ESolveMeasureNormType d)
        : numerator(n), denominator(d) {}
    void set(ESolveMeasureNormType n, ESolveMeasureNormType d) {
        numerator = n;
        denominator = d;
    }
    bool useDefault() const {
        return numerator == SOLVE_MEASURE_ONE && denominator == SOLVE_MEASURE_ONE;
    }
    bool operator()(ESolveMeasureNormType n, ESolveMeasureNormType d) const {
        return numerator == n && denominator == d;
    }
};

struct SolveCriteria {
    static double unspecifiedTolerance() { return -1.0; }
    SolveMeasureType solveMeasureType;
    double requestedTol = unspecifiedTolerance();
    // "Maximum Iterations" (int) here overrides the solver's setting.
    Teuchos::RCP<Teuchos::ParameterList> extraParameters;
    SolveCriteria() = default;
    SolveCriteria(SolveMeasureType m, double tol,
                  const Teuchos::RCP<Teuchos::ParameterList>& extra = Teuchos::null)
        : solveMeasureType(m), requestedTol(tol), extraParameters(extra) {}
};

enum ESolveStatus { SOLVE_STATUS_CONVERGED, SOLVE_STATUS_UNCONVERGED, SOLVE_STATUS_UNKNOWN };

inline const char* toString(ESolveStatus s) {
    switch (s) {
        case SOLVE_STATUS_CONVERGED: return "SOLVE_STATUS_CONVERGED";
        case SOLVE_STATUS_UNCONVERGED: return "SOLVE_STATUS_UNCONVERGED";
        default: return "SOLVE_STATUS_UNKNOWN";
    }
}

struct SolveStatus {
    static double unknownTolerance() { return -1.0; }
    ESolveStatus solveStatus = SOLVE_STATUS_UNKNOWN;
    double achievedTol = unknownTolerance();
    std::string message;
    Teuchos::RCP<Teuchos::ParameterList> extraParameters;
};

// Teuchos::EVerbosityLevel's values; "VerboseObject" -> "Verbosity Level"
// spells them "default", "none", "low", "medium", "high", "extreme".
enum EVerbosityLevel {
    VERB_DEFAULT = -1,
    VERB_NONE = 0,
    VERB_LOW = 1,
    VERB_MEDIUM = 2,
    VERB_HIGH = 3,
    VERB_EXTREME = 4
};

inline EVerbosityLevel verbosityLevel(const std::string& s) {
    static const char* names[] = {"default", "none", "low", "medium", "high", "extreme"};
    for (int i = 0; i < 6; ++i)
        if (s == names[i]) return EVerbosityLevel(i - 1);
    throw Teuchos::Exceptions::InvalidParameterValue("\"Verbosity Level\" = \"" + s +
                                                     "\" is not a verbosity level");
}

// ---------------------------------------------------------------------------
// Blocks of vectors (thyra/src/MCLS_MultiVectorTraits.hpp:95-395)
// ---------------------------------------------------------------------------

template <class MultiVector, class Matrix>
struct MultiVectorTraits;  // specialise for a user's block type

// Host block of vectors: column j is X[j].
typedef std::vector<HostVector> HostMultiVector;

template <>
struct MultiVectorTraits<HostMultiVector, HostCrsMatrix> {
    typedef HostMultiVector multivector_type;
    typedef HostVector vector_type;
    typedef double scalar_type;
    static int getNumVectors(const HostMultiVector& X) { return int(X.size()); }
    // Views of column `id`, valid while X lives.
    static Teuchos::RCP<const HostVector> getVector(const HostMultiVector& X, int id) {
        return Teuchos::rcp(&X.at(size_t(id)), false);
    }
    static Teuchos::RCP<HostVector> getVectorNonConst(HostMultiVector& X, int id) {
        return Teuchos::rcp(&X.at(size_t(id)), false);
    }
};

// ---------------------------------------------------------------------------
// LinearProblemAdapter: A X = B as one LinearProblem per column
// ---------------------------------------------------------------------------

template <class MultiVector, class Matrix>
class LinearProblemAdapter : public virtual Teuchos::Describable {
  public:
    typedef MultiVectorTraits<MultiVector, Matrix> MVT;
    typedef typename MVT::vector_type Vector;
    typedef LinearProblem<Vector, Matrix> Problem;

    LinearProblemAdapter() = default;
    LinearProblemAdapter(const Teuchos::RCP<const Matrix>& A, const Teuchos::RCP<MultiVector>& x,
                         const Teuchos::RCP<const MultiVector>& b)
        : d_A(A), d_x(x), d_b(b) {}

    // Column `id` of X and B with the block's operator and preconditioners.
    // Every call builds a new LinearProblem over the same matrices, so a
    // manager keeps its device domain from one column to the next.
    Teuchos::RCP<Problem> getSubProblem(int id) const {
        if (!Teuchos::nonnull(d_A) || !Teuchos::nonnull(d_x) || !Teuchos::nonnull(d_b))
            throw Assertion("LinearProblemAdapter: operator, LHS and RHS must be set");
        if (id < 0 || id >= getNumSubProblems())
            throw Assertion("LinearProblemAdapter: no sub-problem " + std::to_string(id));
        auto lp = Teuchos::rcp(
            new Problem(d_A, MVT::getVectorNonConst(*d_x, id), MVT::getVector(*d_b, id)));
        if (Teuchos::nonnull(d_PL)) lp->setLeftPrec(d_PL);
        if (Teuchos::nonnull(d_PR)) lp->setRightPrec(d_PR);
        return lp;
    }
    // Columns of X; B must have as many.
    int getNumSubProblems() const {
        if (!Teuchos::nonnull(d_x)) throw Assertion("LinearProblemAdapter: no LHS");
        const int n = MVT::getNumVectors(*d_x);
        if (Teuchos::nonnull(d_b) && MVT::getNumVectors(*d_b) != n)
            throw Assertion("LinearProblemAdapter: LHS and RHS differ in their column counts");
        return n;
    }

    void setOperator(const Teuchos::RCP<const Matrix>& A) { d_A = A; }
    void setLHS(const Teuchos::RCP<MultiVector>& x) { d_x = x; }
    void setRHS(const Teuchos::RCP<const MultiVector>& b) { d_b = b; }
    void releaseLHS() { d_x = Teuchos::null; }
    void releaseRHS() { d_b = Teuchos::null; }
    void setLeftPrec(const Teuchos::RCP<const Matrix>& PL) { d_PL = PL; }
    void setRightPrec(const Teuchos::RCP<const Matrix>& PR) { d_PR = PR; }
    Teuchos::RCP<const Matrix> getOperator() const { return d_A; }
    Teuchos::RCP<MultiVector> getLHS() const { return d_x; }
    Teuchos::RCP<const MultiVector> getRHS() const { return d_b; }
    Teuchos::RCP<const Matrix> getLeftPrec() const { return d_PL; }
    Teuchos::RCP<const Matrix> getRightPrec() const { return d_PR; }

  private:
    Teuchos::RCP<const Matrix> d_A;
    Teuchos::RCP<MultiVector> d_x;
    Teuchos::RCP<const MultiVector> d_b;
    Teuchos::RCP<const Matrix> d_PL;
    Teuchos::RCP<const Matrix> d_PR;
};

// ---------------------------------------------------------------------------
// SolverManagerAdapter: one manager over every column of a block
// ---------------------------------------------------------------------------

template <class MultiVector, class Matrix>
class SolverManagerAdapter : public virtual Teuchos::Describable {
  public:
    typedef typename MultiVectorTraits<MultiVector, Matrix>::vector_type Vector;
    typedef SolverManager<Vector, Matrix> Solver;
    typedef LinearProblemAdapter<MultiVector, Matrix> ProblemAdapter;

    explicit SolverManagerAdapter(const Teuchos::RCP<Solver>& solver) : d_solver(solver) {
        if (!Teuchos::nonnull(solver)) throw Assertion("SolverManagerAdapter: null solver");
    }

    void setProblem(const Teuchos::RCP<ProblemAdapter>& problem) {
        if (!Teuchos::nonnull(problem)) throw Assertion("SolverManagerAdapter: null problem");
        d_problem = problem;
    }
    Teuchos::RCP<ProblemAdapter> getProblem() const { return d_problem; }
    Teuchos::RCP<Solver> getSolver() const { return d_solver; }
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const {
        return d_solver->getValidParameters();
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const {
        return d_solver->getCurrentParameters();
    }
    std::string description() const override { return d_solver->description(); }

    // Solves the columns one after another with `params`: converged when
    // every column converged, the iterations summed, the achieved tolerance
    // the largest (a NaN one is kept).  The extra parameters carry
    // "MCLS/Iteration Count", "Iteration Count" and "MCLS/Achieved Tolerance".
    SolveStatus solve(const Teuchos::RCP<Teuchos::ParameterList>& params) {
        if (!Teuchos::nonnull(d_problem)) throw Assertion("SolverManagerAdapter: no problem set");
        const auto t0 = std::chrono::steady_clock::now();
        bool converged = true;
        int iters = 0;
        double achieved = 0.0;
        const int nprob = d_problem->getNumSubProblems();
        for (int j = 0; j < nprob; ++j) {
            d_solver->setProblem(d_problem->getSubProblem(j));
            d_solver->setParameters(params);
            d_solver->solve();
            iters += d_solver->getNumIters();
            if (!d_solver->getConvergedStatus()) converged = false;
            const double a = double(d_solver->achievedTol());
            if (!(a <= achieved)) achieved = a;
        }
        const double secs =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        SolveStatus st;
        st.solveStatus = converged ? SOLVE_STATUS_CONVERGED : SOLVE_STATUS_UNCONVERGED;
        st.achievedTol = achieved;
        std::ostringstream msg;
        msg << "MCLS solver \"" << d_solver->description() << "\" returned a solve status of \""
            << toString(st.solveStatus) << "\" for " << nprob << " RHSs using " << iters
            << " cumulative iterations for an average of " << (nprob ? iters / nprob : 0)
            << " iterations/RHS and with total CPU time of " << secs << " sec.";
        st.message = msg.str();
        st.extraParameters = Teuchos::parameterList();
        st.extraParameters->set<int>("MCLS/Iteration Count", iters);
        st.extraParameters->set<int>("Iteration Count", iters);
        st.extraParameters->set<double>("MCLS/Achieved Tolerance", achieved);
        return st;
    }

  private:
    Teuchos::RCP<Solver> d_solver;
    Teuchos::RCP<ProblemAdapter> d_problem;
};

// ---------------------------------------------------------------------------
// LinearOpWithSolve: the operator A with solves A X = B
// (thyra/src/Thyra_MCLSLinearOpWithSolve_impl.hpp:52-430)
// ---------------------------------------------------------------------------

template <class MultiVector, class Matrix>
class LinearOpWithSolve : public virtual Teuchos::Describable {
  public:
    typedef MultiVectorTraits<MultiVector, Matrix> MVT;
    typedef typename MVT::vector_type Vector;
    typedef VectorTraits<Vector> VT;
    typedef MatrixTraits<Vector, Matrix> MT;
    typedef LinearProblemAdapter<MultiVector, Matrix> ProblemAdapter;
    typedef SolverManagerAdapter<MultiVector, Matrix> SolverAdapter;
    typedef Preconditioner<Matrix> Prec;

    LinearOpWithSolve() = default;

    // The default tolerance is the solver list's "Convergence Tolerance",
    // else the manager's valid default; a manager without one ("Adjoint MC",
    // "Forward MC") has none, and its solves set no tolerance.
    void initialize(const Teuchos::RCP<ProblemAdapter>& problem,
                    const Teuchos::RCP<Teuchos::ParameterList>& solver_params,
                    const Teuchos::RCP<SolverAdapter>& solver,
                    const Teuchos::RCP<Prec>& prec = Teuchos::null, bool is_external_prec = false,
                    const Teuchos::RCP<const Matrix>& approx_op = Teuchos::null,
                    ESupportSolveUse support_solve_use = SUPPORT_SOLVE_UNSPECIFIED) {
        if (!Teuchos::nonnull(solver) || !Teuchos::nonnull(problem) ||
            !Teuchos::nonnull(problem->getOperator()))
            throw Assertion("LinearOpWithSolve: solver, problem and operator must be set");
        d_problem = problem;
        d_plist = solver_params;
        d_solver = solver;
        d_prec = prec;
        d_is_external_prec = is_external_prec;
        d_approx_op = approx_op;
        d_support_solve_use = support_solve_use;
        d_default_tol = SolveCriteria::unspecifiedTolerance();
        const auto valid = solver->getValidParameters();
        if (Teuchos::nonnull(d_plist) && d_plist->isParameter("Convergence Tolerance"))
            d_default_tol = d_plist->template get<double>("Convergence Tolerance");
        else if (valid->isParameter("Convergence Tolerance"))
            d_default_tol = valid->template get<double>("Convergence Tolerance");
    }
    void uninitialize(Teuchos::RCP<ProblemAdapter>* problem = nullptr,
                      Teuchos::RCP<Teuchos::ParameterList>* solver_params = nullptr,
                      Teuchos::RCP<SolverAdapter>* solver = nullptr,
                      Teuchos::RCP<Prec>* prec = nullptr, bool* is_external_prec = nullptr,
                      Teuchos::RCP<const Matrix>* approx_op = nullptr,
                      ESupportSolveUse* support_solve_use = nullptr) {
        if (problem) *problem = d_problem;
        if (solver_params) *solver_params = d_plist;
        if (solver) *solver = d_solver;
        if (prec) *prec = d_prec;
        if (is_external_prec) *is_external_prec = d_is_external_prec;
        if (approx_op) *approx_op = d_approx_op;
        if (support_solve_use) *support_solve_use = d_support_solve_use;
        *this = LinearOpWithSolve();
    }
    bool isInitialized() const { return Teuchos::nonnull(d_solver); }

    Teuchos::RCP<ProblemAdapter> problem() const { return d_problem; }
    Teuchos::RCP<SolverAdapter> solver() const { return d_solver; }
    Teuchos::RCP<Prec> prec() const { return d_prec; }
    bool isExternalPrec() const { return d_is_external_prec; }
    Teuchos::RCP<const Matrix> approxOp() const { return d_approx_op; }
    ESupportSolveUse supportSolveUse() const { return d_support_solve_use; }
    double defaultTolerance() const { return d_default_tol; }

    // Range and domain dimension (square operators only).
    std::int64_t dim() const {
        requireInitialized();
        return MT::getGlobalNumRows(*d_problem->getOperator());
    }

    void setVerbLevel(EVerbosityLevel v) { d_verb = v; }
    EVerbosityLevel getVerbLevel() const { return d_verb; }
    void setOStream(std::ostream* out) {
        d_out = out;
        d_out_owner.reset();
    }
    // A stream the op shares with its creator ("Output File").
    void setOStream(const std::shared_ptr<std::ostream>& out) {
        d_out_owner = out;
        d_out = out.get();
    }

    // Forward solves only, with the solver's own test or the MCSA measure
    // |PL (b - A x)| / |PL b|, requested as NORM_RESIDUAL / NORM_RHS.
    bool solveSupports(EOpTransp trans, const SolveCriteria* criteria = nullptr) const {
        if (trans != NOTRANS) return false;
        if (criteria == nullptr) return true;
        return criteria->solveMeasureType.useDefault() ||
               criteria->solveMeasureType(SOLVE_MEASURE_NORM_RESIDUAL, SOLVE_MEASURE_NORM_RHS);
    }
    bool solveSupportsSolveMeasureType(EOpTransp trans, const SolveMeasureType& m) const {
        SolveCriteria c(m, SolveCriteria::unspecifiedTolerance());
        return solveSupports(trans, &c);
    }

    // Solves A X = B column by column, X holding the initial guesses.  The
    // solver's current parameters are copied, and the copy gets the
    // tolerance (the requested one unless the measure is the default or the
    // tolerance unspecified; the default tolerance otherwise) and the
    // criteria's "Maximum Iterations".  X and B are released afterwards.
    SolveStatus solve(EOpTransp trans, const MultiVector& B, MultiVector* X,
                      const SolveCriteria* criteria = nullptr) const {
        requireInitialized();
        if (trans != NOTRANS) throw Assertion("Solve does not support transpose type.");
        if (!solveSupports(trans, criteria))
            throw Assertion("Solve does not support the requested solve measure.");
        if (X == nullptr) throw Assertion("LinearOpWithSolve::solve: null LHS");
        const auto t0 = std::chrono::steady_clock::now();
        if (d_out && d_verb > VERB_NONE)
            *d_out << "\nSolving block system using MCLS ...\n\n" << std::flush;
        auto tmp = Teuchos::parameterList();
        const auto current = d_solver->getCurrentParameters();
        if (Teuchos::nonnull(current)) tmp->setParameters(*current);
        double tol = d_default_tol;
        if (criteria != nullptr) {
            if (!criteria->solveMeasureType.useDefault() &&
                criteria->requestedTol != SolveCriteria::unspecifiedTolerance())
                tol = criteria->requestedTol;
            const auto& extra = criteria->extraParameters;
            if (Teuchos::nonnull(extra) && extra->template isType<int>("Maximum Iterations"))
                tmp->set<int>("Maximum Iterations", extra->template get<int>("Maximum Iterations"));
        }
        if (tol != SolveCriteria::unspecifiedTolerance())
            tmp->set<double>("Convergence Tolerance", tol);
        d_problem->setLHS(Teuchos::rcp(X, false));
        d_problem->setRHS(Teuchos::rcp(&B, false));
        SolveStatus st;
        try {
            st = d_solver->solve(tmp);
        } catch (...) {
            d_problem->releaseLHS();
            d_problem->releaseRHS();
            throw;
        }
        d_problem->releaseLHS();
        d_problem->releaseRHS();
        if (d_out && d_verb >= VERB_LOW)
            *d_out << "\nTotal solve time = "
                   << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
                   << " sec\n"
                   << std::flush;
        return st;
    }

    // Y = alpha A X + beta Y (the forward operator; beta = 0 overwrites Y).
    bool opSupported(EOpTransp trans) const { return trans == NOTRANS; }
    void apply(EOpTransp trans, const MultiVector& X, MultiVector* Y, double alpha = 1.0,
               double beta = 0.0) const {
        requireInitialized();
        if (trans != NOTRANS) throw Assertion("LinearOpWithSolve::apply: forward operator only");
        if (Y == nullptr || MVT::getNumVectors(X) != MVT::getNumVectors(*Y))
            throw Assertion("LinearOpWithSolve::apply: X and Y differ in their column counts");
        const Matrix& A = *d_problem->getOperator();
        for (int j = 0; j < MVT::getNumVectors(X); ++j) {
            auto x = MVT::getVector(X, j);
            auto y = MVT::getVectorNonConst(*Y, j);
            auto ax = VT::clone(*x);
            MT::apply(A, *x, *ax);
            const std::int64_t n = VT::getGlobalLength(*y);
            if (VT::getGlobalLength(*ax) != n)
                throw Assertion("LinearOpWithSolve::apply: Y has the wrong length");
            const double* a = VT::view(*ax);
            double* yv = VT::viewNonConst(*y);
            for (std::int64_t i = 0; i < n; ++i)
                yv[i] = beta == 0.0 ? alpha * a[i] : alpha * a[i] + beta * yv[i];
        }
    }

    std::string description() const override {
        std::ostringstream s;
        s << "MCLS::LinearOpWithSolve";
        if (isInitialized()) {
            s << "{iterativeSolver='" << d_solver->description() << "',dim=" << dim();
            if (Teuchos::nonnull(d_problem->getLeftPrec())) s << ",leftPrecOp";
            if (Teuchos::nonnull(d_problem->getRightPrec())) s << ",rightPrecOp";
            s << "}";
        }
        return s.str();
    }

  private:
    void requireInitialized() const {
        if (!isInitialized()) throw Assertion("LinearOpWithSolve: not initialized");
    }

    Teuchos::RCP<ProblemAdapter> d_problem;
    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    Teuchos::RCP<SolverAdapter> d_solver;
    Teuchos::RCP<Prec> d_prec;
    bool d_is_external_prec = false;
    Teuchos::RCP<const Matrix> d_approx_op;
    ESupportSolveUse d_support_solve_use = SUPPORT_SOLVE_UNSPECIFIED;
    double d_default_tol = SolveCriteria::unspecifiedTolerance();
    EVerbosityLevel d_verb = VERB_DEFAULT;
    std::ostream* d_out = nullptr;
    std::shared_ptr<std::ostream> d_out_owner;
};

// ---------------------------------------------------------------------------
// LinearOpWithSolveFactory
// (thyra/src/Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:58-615)
// ---------------------------------------------------------------------------

template <class MultiVector, class Matrix>
class LinearOpWithSolveFactory : public virtual Teuchos::Describable {
  public:
    typedef MultiVectorTraits<MultiVector, Matrix> MVT;
    typedef typename MVT::vector_type Vector;
    typedef MatrixTraits<Vector, Matrix> MT;
    typedef LinearOpWithSolve<MultiVector, Matrix> Op;
    typedef LinearProblemAdapter<MultiVector, Matrix> ProblemAdapter;
    typedef SolverManagerAdapter<MultiVector, Matrix> SolverAdapter;
    typedef PreconditionerFactoryBase<Matrix> PrecFactory;
    typedef Preconditioner<Matrix> Prec;

    static constexpr const char* SolverType_name = "Solver Type";
    static constexpr const char* SolverType_default = "MCSA";
    static constexpr const char* SolverTypes_name = "Solver Types";
    static constexpr const char* ConvergenceTestFrequency_name = "Convergence Test Frequency";

    // "Solver Type" values: the reference's five, then the SolverFactory
    // names that also pick the Monte Carlo direction.
    static const std::vector<std::string>& solverTypeNames() {
        static const std::vector<std::string> names = {
            "MCSA",         "Adjoint MC",   "Forward MC",       "Fixed Point",     "Anderson",
            "Adjoint MCSA", "Forward MCSA", "Adjoint Anderson", "Forward Anderson"};
        return names;
    }
    // The SolverFactory name a "Solver Type" creates.
    static std::string managerName(const std::string& solver_type) {
        if (solver_type == "MCSA") return "Adjoint MCSA";
        if (solver_type == "Anderson") return "Adjoint Anderson";
        return solver_type;
    }

    LinearOpWithSolveFactory() : d_valid(makeValidParameters()) {}
    explicit LinearOpWithSolveFactory(const Teuchos::RCP<PrecFactory>& prec_factory)
        : LinearOpWithSolveFactory() {
        setPreconditionerFactory(prec_factory, "");
    }

    // ---- parameters ----

    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const { return d_valid; }

    // Validates the list one sublist level deep against getValidParameters()
    // and fills in what is missing (Teuchos::Exceptions::InvalidParameterName
    // / InvalidParameterType); an unknown "Solver Type" or "Verbosity Level"
    // throws InvalidParameterValue.  The solvers created afterwards take
    // their parameters from this list's "Solver Types" sublist of the chosen
    // type, by reference.
    void setParameterList(const Teuchos::RCP<Teuchos::ParameterList>& params) {
        if (!Teuchos::nonnull(params))
            throw Assertion("LinearOpWithSolveFactory: null parameter list");
        params->validateParametersAndSetDefaults(*d_valid, 1);
        const std::string type = params->template get<std::string>(SolverType_name);
        bool known = false;
        for (const auto& n : solverTypeNames()) known = known || n == type;
        if (!known)
            throw Teuchos::Exceptions::InvalidParameterValue(
                std::string("\"") + SolverType_name + "\" = \"" + type +
                "\" is not one of the MCLS solver types");
        const auto& vo = params->sublist("VerboseObject");
        const EVerbosityLevel verb =
            verbosityLevel(vo.template get<std::string>("Verbosity Level"));
        const std::string file = vo.template get<std::string>("Output File");
        std::shared_ptr<std::ofstream> out_file;
        if (file != "none") {
            out_file = std::make_shared<std::ofstream>(file);
            if (!*out_file)
                throw Teuchos::Exceptions::InvalidParameterValue("\"Output File\" = \"" + file +
                                                                 "\" cannot be opened");
        }
        d_plist = params;
        d_solver_type = type;
        d_convergence_test_frequency =
            params->template get<int>(ConvergenceTestFrequency_name);
        d_verb = verb;
        if (out_file) {
            d_out_file = out_file;
            d_out = out_file.get();
        }
    }
    Teuchos::RCP<Teuchos::ParameterList> getNonconstParameterList() { return d_plist; }
    Teuchos::RCP<const Teuchos::ParameterList> getParameterList() const { return d_plist; }
    Teuchos::RCP<Teuchos::ParameterList> unsetParameterList() {
        auto p = d_plist;
        d_plist = Teuchos::null;
        d_solver_type = SolverType_default;
        d_convergence_test_frequency = 1;
        d_verb = VERB_DEFAULT;
        return p;
    }
    const std::string& solverType() const { return d_solver_type; }
    int convergenceTestFrequency() const { return d_convergence_test_frequency; }

    void setVerbLevel(EVerbosityLevel v) { d_verb = v; }
    EVerbosityLevel getVerbLevel() const { return d_verb; }
    void setOStream(std::ostream* out) {
        d_out = out;
        d_out_file.reset();
    }

    // ---- preconditioner factory ----

    bool acceptsPreconditionerFactory() const { return true; }
    void setPreconditionerFactory(const Teuchos::RCP<PrecFactory>& f, const std::string& name) {
        d_prec_factory = f;
        d_prec_factory_name = name;
    }
    Teuchos::RCP<PrecFactory> getPreconditionerFactory() const { return d_prec_factory; }
    void unsetPreconditionerFactory(Teuchos::RCP<PrecFactory>* f = nullptr,
                                    std::string* name = nullptr) {
        if (f) *f = d_prec_factory;
        if (name) *name = d_prec_factory_name;
        d_prec_factory = Teuchos::null;
        d_prec_factory_name = "";
    }
    bool supportsPreconditionerInputType(EPreconditionerInputType t) const {
        return Teuchos::nonnull(d_prec_factory) || t == PRECONDITIONER_INPUT_TYPE_AS_OPERATOR;
    }

    // ---- operators ----

    bool isCompatible(const Matrix& A) const {
        const bool prec_ok = !Teuchos::nonnull(d_prec_factory) || d_prec_factory->isCompatible(A);
        return prec_ok && MT::getGlobalNumRows(A) > 0;
    }
    Teuchos::RCP<Op> createOp() const { return Teuchos::rcp(new Op()); }

    // A alone, with the preconditioner factory's preconditioner when one is
    // set (built anew).
    void initializeOp(const Teuchos::RCP<const Matrix>& A, Op* op,
                      ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const {
        selectOp(A, Teuchos::null, Teuchos::null, false, op, use);
    }
    // As initializeOp, keeping the preconditioner the factory built for op
    // earlier instead of rebuilding it.
    void initializeAndReuseOp(const Teuchos::RCP<const Matrix>& A, Op* op) const {
        selectOp(A, Teuchos::null, Teuchos::null, true, op, SUPPORT_SOLVE_UNSPECIFIED);
    }
    // With a caller's built preconditioner (its left and right matrices).
    void initializePreconditionedOp(const Teuchos::RCP<const Matrix>& A,
                                    const Teuchos::RCP<Prec>& prec, Op* op,
                                    ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const {
        selectOp(A, Teuchos::null, prec, false, op, use);
    }
    // With left and right preconditioner matrices built elsewhere (either
    // may be null), as a GivenPreconditioner.
    void initializePreconditionedOp(const Teuchos::RCP<const Matrix>& A,
                                    const Teuchos::RCP<const Matrix>& PL,
                                    const Teuchos::RCP<const Matrix>& PR, Op* op,
                                    ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const {
        selectOp(A, Teuchos::null, Teuchos::rcp(new GivenPreconditioner<Matrix>(PL, PR)), false,
                 op, use);
    }
    // The factory's preconditioner built from approx_A instead of A.
    void initializeApproxPreconditionedOp(const Teuchos::RCP<const Matrix>& A,
                                          const Teuchos::RCP<const Matrix>& approx_A, Op* op,
                                          ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const {
        selectOp(A, approx_A, Teuchos::null, false, op, use);
    }
    void uninitializeOp(Op* op, Teuchos::RCP<const Matrix>* A = nullptr,
                        Teuchos::RCP<Prec>* prec = nullptr,
                        Teuchos::RCP<const Matrix>* approx_A = nullptr,
                        ESupportSolveUse* use = nullptr) const {
        if (op == nullptr) throw Assertion("LinearOpWithSolveFactory::uninitializeOp: null op");
        Teuchos::RCP<ProblemAdapter> lp;
        Teuchos::RCP<Prec> p;
        bool external = false;
        op->uninitialize(&lp, nullptr, nullptr, &p, &external, approx_A, use);
        if (A) *A = Teuchos::nonnull(lp) ? lp->getOperator() : Teuchos::null;
        if (prec) *prec = external ? p : Teuchos::null;
    }

    std::string description() const override { return "MCLS::LinearOpWithSolveFactory"; }

  private:
    // Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:424-521: the
    // preconditioner (given, reused or built by the factory), then the
    // problem adapter and the manager of the selected type.
    void selectOp(const Teuchos::RCP<const Matrix>& A, const Teuchos::RCP<const Matrix>& approx_A,
                  const Teuchos::RCP<Prec>& prec_in, bool reuse_prec, Op* op,
                  ESupportSolveUse use) const {
        if (op == nullptr || !Teuchos::nonnull(A))
            throw Assertion("LinearOpWithSolveFactory: null operator or op");
        if (d_out && d_verb > VERB_LOW)
            *d_out << "\nEntering MCLS::LinearOpWithSolveFactory::initializeOp(...) ...\n"
                   << std::flush;
        Teuchos::RCP<Prec> prec = prec_in;
        bool external = Teuchos::nonnull(prec_in);
        if (!external && Teuchos::nonnull(d_prec_factory)) {
            Teuchos::RCP<Prec> mine = op->isExternalPrec() ? Teuchos::null : op->prec();
            const bool existing = Teuchos::nonnull(mine);
            if (!existing) mine = d_prec_factory->createPrec();
            if (!(existing && reuse_prec))
                d_prec_factory->initializePrec(Teuchos::nonnull(approx_A) ? approx_A : A,
                                               mine.get());
            prec = mine;
        }
        auto lp = Teuchos::rcp(new ProblemAdapter());
        lp->setOperator(A);
        if (Teuchos::nonnull(prec)) {
            lp->setLeftPrec(prec->getLeftPreconditioner());
            lp->setRightPrec(prec->getRightPreconditioner());
        }
        auto solver_params =
            Teuchos::nonnull(d_plist)
                ? Teuchos::sublist(Teuchos::sublist(d_plist, SolverTypes_name), d_solver_type)
                : Teuchos::parameterList();
        auto manager = SolverFactory<Vector, Matrix>().create(managerName(d_solver_type),
                                                              solver_params);
        auto solver = Teuchos::rcp(new SolverAdapter(manager));
        solver->setProblem(lp);
        op->initialize(lp, solver_params, solver, prec, external, approx_A, use);
        if (d_out_file)
            op->setOStream(std::shared_ptr<std::ostream>(d_out_file));
        else
            op->setOStream(d_out);
        op->setVerbLevel(d_verb);
        if (d_out && d_verb > VERB_LOW)
            *d_out << "\nLeaving MCLS::LinearOpWithSolveFactory::initializeOp(...) ...\n"
                   << std::flush;
    }

    // Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:367-420: each "Solver
    // Types" sublist holds the valid parameters of its manager.
    static Teuchos::RCP<const Teuchos::ParameterList> makeValidParameters() {
        auto pl = Teuchos::parameterList("MCLSLinearOpWithSolveFactory");
        pl->set<std::string>(SolverType_name, SolverType_default);
        pl->set<int>(ConvergenceTestFrequency_name, 1);
        Teuchos::ParameterList& types = pl->sublist(SolverTypes_name);
        SolverFactory<Vector, Matrix> factory;
        for (const auto& name : solverTypeNames())
            types.sublist(name).setParameters(
                *factory.create(managerName(name), Teuchos::parameterList())->getValidParameters());
        Teuchos::ParameterList& verbose = pl->sublist("VerboseObject");
        verbose.set<std::string>("Verbosity Level", "default");
        verbose.set<std::string>("Output File", "none");
        return pl;
    }

    Teuchos::RCP<const Teuchos::ParameterList> d_valid;
    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    std::string d_solver_type = SolverType_default;
    int d_convergence_test_frequency = 1;
    Teuchos::RCP<PrecFactory> d_prec_factory;
    std::string d_prec_factory_name;
    EVerbosityLevel d_verb = VERB_DEFAULT;
    std::ostream* d_out = nullptr;
    std::shared_ptr<std::ofstream> d_out_file;  // "Output File", when not "none"
};

}  // namespace MCLS

#endif  // MCLS_LINEAROPWITHSOLVE_HPP
