// LinearOpWithSolve test: the Stratimikos-facing solver
// (include/MCLS_LinearOpWithSolve.hpp, include/MCLS_PreconditionerFactory.hpp).
//
//   lows_test cpu DIR   no device: the factory's parameter lists and their
//                       validation, "Solver Type" -> manager, the solve
//                       vocabulary, and the column loop, tolerance handling
//                       and status over a host Jacobi solver plugged in behind
//                       the SolverManager interface; DIR takes an output file.
//   lows_test gpu       blocks of right-hand sides solved on the device
//                       through the factory ("MCSA", "Fixed Point",
//                       "Anderson", the "Point Jacobi" preconditioner
//                       factory), after the reference's LOWS test
//                       (thyra/test/LOWSFactoryTpetra/test_single_mcls_thyra_solver.cpp:
//                       forward solves of several right-hand sides, residual
//                       and solution checked per column).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "MCLS_LinearOpWithSolve.hpp"

typedef MCLS::HostVector Vec;
typedef MCLS::HostCrsMatrix Mat;
typedef MCLS::HostMultiVector MV;
typedef MCLS::LinearOpWithSolveFactory<MV, Mat> Factory;
typedef MCLS::LinearOpWithSolve<MV, Mat> Lows;
typedef Teuchos::ParameterList PL;

static int g_failures = 0;
static std::string g_section = "start";
#define EXPECT(cond)                                                                       \
    do {                                                                                   \
        if (!(cond)) {                                                                     \
            std::printf("FAILED [%s] %s:%d: %s\n", g_section.c_str(), __FILE__, __LINE__, \
                        #cond);                                                            \
            ++g_failures;                                                                  \
        }                                                                                  \
    } while (0)

template <class E, class F>
static bool throws(F&& f, const char* needle = nullptr) {
    try {
        f();
    } catch (const E& e) {
        return needle == nullptr || std::string(e.what()).find(needle) != std::string::npos;
    } catch (...) {
        return false;
    }
    return false;
}

// Tridiagonal (-0.14, 1, -0.14) with the explicit zeros of the reference's
// manager tests.
static Teuchos::RCP<Mat> tridiag(int n) {
    auto A = Teuchos::rcp(new Mat);
    A->n = n;
    A->rowptr.assign(1, 0);
    for (int i = 0; i < n; ++i) {
        int c0 = i == 0 ? 0 : (i == n - 1 ? n - 3 : i - 1);
        for (int c = c0; c < c0 + 3; ++c) {
            A->colind.push_back(c);
            A->values.push_back(c == i ? 1.0 : (std::abs(c - i) == 1 ? -0.14 : 0.0));
        }
        A->rowptr.push_back(std::int64_t(A->colind.size()));
    }
    return A;
}

// The fixed-point manager test's operator
// (tpetra/test/tstTpetraFixedPointSolverManager.cpp:72-120).
static Teuchos::RCP<Mat> fixed_point_matrix(int n) {
    auto F = Teuchos::rcp(new Mat);
    F->n = n;
    F->rowptr.assign(1, 0);
    for (int i = 0; i < n; ++i) {
        const int c0 = i == 0 ? 0 : (i == n - 1 ? n - 3 : i - 1);
        const double v[3] = {0.14, i == 0 || i == n - 1 ? 0.14 : 1.0,
                             i == 0 || i == n - 1 ? 1.0 : 0.14};
        for (int k = 0; k < 3; ++k) {
            F->colind.push_back(c0 + k);
            F->values.push_back(v[k]);
        }
        F->rowptr.push_back(std::int64_t(F->colind.size()));
    }
    return F;
}

static Vec direct(const Mat& A, const Vec& b) {
    const int n = int(A.n);
    std::vector<double> M(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (auto p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p)
            M[size_t(i) * n + A.colind[p]] += A.values[p];
    Vec x = b;
    for (int k = 0; k < n; ++k)
        for (int i = k + 1; i < n; ++i) {
            double f = M[size_t(i) * n + k] / M[size_t(k) * n + k];
            for (int j = k; j < n; ++j) M[size_t(i) * n + j] -= f * M[size_t(k) * n + j];
            x[i] -= f * x[k];
        }
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) x[i] -= M[size_t(i) * n + j] * x[j];
        x[i] /= M[size_t(i) * n + i];
    }
    return x;
}

static double rel_err(const Vec& a, const Vec& b) {
    double d = 0, n = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        d += (a[i] - b[i]) * (a[i] - b[i]);
        n += b[i] * b[i];
    }
    return std::sqrt(d / n);
}

// |b - A x|_2 / |b|_2
static double rel_residual(const Mat& A, const Vec& x, const Vec& b) {
    Vec ax;
    MCLS::MatrixTraits<Vec, Mat>::apply(A, x, ax);
    double r = 0, s = 0;
    for (size_t i = 0; i < b.size(); ++i) {
        r += (b[i] - ax[i]) * (b[i] - ax[i]);
        s += b[i] * b[i];
    }
    return std::sqrt(r / s);
}

// Jacobi iteration on the host behind the SolverManager interface, so the
// adapter's logic can be checked without a device.  It records the
// tolerance and iteration limit of every solve and whether the problem
// carried preconditioners.
class HostJacobi : public MCLS::SolverManager<Vec, Mat> {
  public:
    typedef MCLS::LinearProblem<Vec, Mat> LP;

    explicit HostJacobi(const Teuchos::RCP<PL>& pl) : d_pl(pl) {}
    const LP& getProblem() const override { return *d_lp; }
    Teuchos::RCP<const PL> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<double>("Convergence Tolerance", 1.0e-6);
        pl->set<int>("Maximum Iterations", 1000);
        return pl;
    }
    Teuchos::RCP<const PL> getCurrentParameters() const override { return d_pl; }
    double achievedTol() const override { return d_achieved; }
    int getNumIters() const override { return d_iters; }
    void setProblem(const Teuchos::RCP<LP>& p) override { d_lp = p; }
    void setParameters(const Teuchos::RCP<PL>& p) override { d_pl = p; }
    bool solve() override {
        const double tol = d_pl->isParameter("Convergence Tolerance")
                               ? d_pl->get<double>("Convergence Tolerance")
                               : 1.0e-6;
        const int maxit =
            d_pl->isParameter("Maximum Iterations") ? d_pl->get<int>("Maximum Iterations") : 1000;
        tolerances.push_back(tol);
        limits.push_back(maxit);
        with_left.push_back(d_lp->isLeftPrec());
        const Mat& A = *d_lp->getOperator();
        Vec& x = *d_lp->getLHS();
        const Vec& b = *d_lp->getRHS();
        Vec diag(b.size(), 0.0);
        for (std::int64_t i = 0; i < A.n; ++i)
            for (auto p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p)
                if (A.colind[p] == i) diag[size_t(i)] += A.values[p];
        d_iters = 0;
        d_achieved = rel_residual(A, x, b);
        while (d_achieved > tol && d_iters < maxit) {
            Vec ax;
            MCLS::MatrixTraits<Vec, Mat>::apply(A, x, ax);
            for (size_t i = 0; i < x.size(); ++i) x[i] += (b[i] - ax[i]) / diag[i];
            ++d_iters;
            d_achieved = rel_residual(A, x, b);
        }
        d_conv = d_achieved <= tol;
        return d_conv;
    }
    bool getConvergedStatus() const override { return d_conv; }
    std::string description() const override { return "host Jacobi"; }

    std::vector<double> tolerances;
    std::vector<int> limits;
    std::vector<bool> with_left;

  private:
    Teuchos::RCP<PL> d_pl;
    Teuchos::RCP<LP> d_lp;
    double d_achieved = 0.0;
    int d_iters = 0;
    bool d_conv = false;
};

// A LOWS over HostJacobi, assembled the way the factory assembles its own.
static Teuchos::RCP<Lows> host_lows(const Teuchos::RCP<const Mat>& A,
                                    const Teuchos::RCP<PL>& solver_pl,
                                    Teuchos::RCP<HostJacobi>* solver_out,
                                    const Teuchos::RCP<const Mat>& PL_ = Teuchos::null) {
    auto solver = Teuchos::rcp(new HostJacobi(solver_pl));
    auto lp = Teuchos::rcp(new MCLS::LinearProblemAdapter<MV, Mat>());
    lp->setOperator(A);
    lp->setLeftPrec(PL_);
    auto adapter = Teuchos::rcp(new MCLS::SolverManagerAdapter<MV, Mat>(solver));
    adapter->setProblem(lp);
    auto op = Teuchos::rcp(new Lows());
    op->initialize(lp, solver_pl, adapter);
    if (solver_out) *solver_out = solver;
    return op;
}

// Host diagonal-inverse preconditioner and a factory that counts its builds.
class HostDiagPrec : public MCLS::Preconditioner<Mat> {
  public:
    Teuchos::RCP<const PL> getValidParameters() const override { return Teuchos::parameterList(); }
    Teuchos::RCP<const PL> getCurrentParameters() const override { return Teuchos::parameterList(); }
    void setParameters(const Teuchos::RCP<PL>&) override {}
    void setOperator(const Teuchos::RCP<const Mat>& A) override { d_A = A; }
    const Mat& getOperator() const override { return *d_A; }
    void buildPreconditioner() override {
        auto M = Teuchos::rcp(new Mat);
        M->n = d_A->n;
        for (std::int64_t i = 0; i < d_A->n; ++i) {
            double d = 0.0;
            for (auto p = d_A->rowptr[i]; p < d_A->rowptr[i + 1]; ++p)
                if (d_A->colind[p] == i) d += d_A->values[p];
            M->colind.push_back(i);
            M->values.push_back(1.0 / d);
            M->rowptr.push_back(i + 1);
        }
        d_M = M;
    }
    Teuchos::RCP<const Mat> getLeftPreconditioner() const override { return d_M; }
    Teuchos::RCP<const Mat> getRightPreconditioner() const override { return Teuchos::null; }

  private:
    Teuchos::RCP<const Mat> d_A, d_M;
};

class CountingPrecFactory : public MCLS::PreconditionerFactoryBase<Mat> {
  public:
    bool isCompatible(const Mat& A) const override { return A.n > 0; }
    Teuchos::RCP<Prec> createPrec() const override {
        ++created;
        return Teuchos::rcp(new HostDiagPrec());
    }
    void initializePrec(const Teuchos::RCP<const Mat>& A, Prec* prec) const override {
        ++built;
        last_operator = A.get();
        prec->setOperator(A);
        prec->buildPreconditioner();
    }
    mutable int created = 0, built = 0;
    mutable const Mat* last_operator = nullptr;
};

static MV block(int n, std::initializer_list<double> values) {
    MV B;
    for (double v : values) B.push_back(Vec(size_t(n), v));
    return B;
}

static void cpu_checks(const std::string& dir) {
    const int n = 10;
    auto A = tridiag(n);

    g_section = "solve vocabulary";
    {
        MCLS::SolveMeasureType m;
        EXPECT(m.useDefault());
        m.set(MCLS::SOLVE_MEASURE_NORM_RESIDUAL, MCLS::SOLVE_MEASURE_NORM_RHS);
        EXPECT(!m.useDefault() &&
               m(MCLS::SOLVE_MEASURE_NORM_RESIDUAL, MCLS::SOLVE_MEASURE_NORM_RHS));
        MCLS::SolveCriteria c;
        EXPECT(c.requestedTol == MCLS::SolveCriteria::unspecifiedTolerance());
        MCLS::SolveStatus s;
        EXPECT(s.solveStatus == MCLS::SOLVE_STATUS_UNKNOWN &&
               s.achievedTol == MCLS::SolveStatus::unknownTolerance());
        EXPECT(std::string(MCLS::toString(MCLS::SOLVE_STATUS_CONVERGED)) ==
               "SOLVE_STATUS_CONVERGED");
        EXPECT(MCLS::verbosityLevel("extreme") == MCLS::VERB_EXTREME &&
               MCLS::verbosityLevel("default") == MCLS::VERB_DEFAULT);
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterValue>(
            [] { MCLS::verbosityLevel("loud"); }));
    }

    g_section = "factory valid parameters";
    {
        Factory f;
        auto v = f.getValidParameters();
        EXPECT(v->get<std::string>("Solver Type") == "MCSA");
        EXPECT(v->get<int>("Convergence Test Frequency") == 1);
        const PL& types = v->sublist("Solver Types");
        for (const auto& name : Factory::solverTypeNames()) EXPECT(types.isSublist(name));
        EXPECT(types.sublist("MCSA").get<double>("Convergence Tolerance") == 1.0);
        EXPECT(types.sublist("MCSA").get<std::string>("Fixed Point Type") == "Richardson");
        EXPECT(types.sublist("MCSA").isParameter("Sample Ratio"));
        EXPECT(types.sublist("Adjoint MC").isParameter("History Length"));
        EXPECT(!types.sublist("Adjoint MC").isParameter("Convergence Tolerance"));
        EXPECT(types.sublist("Fixed Point").get<double>("Richardson Relaxation") == 1.0);
        EXPECT(types.sublist("Anderson").sublist("Anderson Parameters").get<int>(
                   "Storage Depth") == 2);
        EXPECT(v->sublist("VerboseObject").get<std::string>("Verbosity Level") == "default");
        EXPECT(f.acceptsPreconditionerFactory());
        EXPECT(f.supportsPreconditionerInputType(MCLS::PRECONDITIONER_INPUT_TYPE_AS_OPERATOR));
        EXPECT(!f.supportsPreconditionerInputType(MCLS::PRECONDITIONER_INPUT_TYPE_AS_MATRIX));
        EXPECT(f.isCompatible(*A));
        EXPECT(f.description() == "MCLS::LinearOpWithSolveFactory");
    }

    g_section = "factory parameter validation";
    {
        Factory f;
        auto pl = Teuchos::parameterList();
        f.setParameterList(pl);  // an empty list takes every default
        EXPECT(pl->get<std::string>("Solver Type") == "MCSA");
        EXPECT(pl->sublist("Solver Types").sublist("Forward MC").isParameter("Sample Ratio"));
        EXPECT(f.solverType() == "MCSA" && f.convergenceTestFrequency() == 1);
        EXPECT(f.getParameterList() == pl && f.getNonconstParameterList() == pl);

        // The reference's own LOWS list: the MCSA sublist keeps the user's
        // keys, including ones the GPU managers accept and ignore.
        auto ref = Teuchos::parameterList();
        ref->set<std::string>("Solver Type", "Fixed Point");
        PL& mcsa = ref->sublist("Solver Types").sublist("MCSA");
        mcsa.set<int>("Maximum Iterations", 40);
        mcsa.set<double>("Convergence Tolerance", 1.0e-8);
        mcsa.set<std::string>("MC Type", "Adjoint");
        mcsa.set<int>("Overlap Size", 0);
        ref->sublist("Solver Types").sublist("Fixed Point").set<double>("Richardson Relaxation",
                                                                        0.9);
        ref->set<int>("Convergence Test Frequency", 3);
        f.setParameterList(ref);
        EXPECT(f.solverType() == "Fixed Point" && f.convergenceTestFrequency() == 3);
        EXPECT(mcsa.get<int>("Maximum Iterations") == 40 && mcsa.isParameter("MC Type"));
        EXPECT(!mcsa.isParameter("History Length"));  // sublists of "Solver Types" are not filled
        EXPECT(ref->sublist("Solver Types").sublist("Anderson").isSublist("Anderson Parameters"));
        EXPECT(f.unsetParameterList() == ref && f.solverType() == "MCSA");

        auto bad_type = Teuchos::parameterList();
        bad_type->set<std::string>("Solver Type", "GMRES");
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterValue>(
            [&] { f.setParameterList(bad_type); }, "GMRES"));
        auto bad_name = Teuchos::parameterList();
        bad_name->set<int>("Krylov Length", 30);
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterName>(
            [&] { f.setParameterList(bad_name); }, "Krylov Length"));
        auto bad_kind = Teuchos::parameterList();
        bad_kind->set<double>("Convergence Test Frequency", 2.0);
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterType>(
            [&] { f.setParameterList(bad_kind); }));
        auto bad_sub = Teuchos::parameterList();
        bad_sub->sublist("Solver Types").sublist("Belos");
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterName>(
            [&] { f.setParameterList(bad_sub); }, "Belos"));
        auto bad_verb = Teuchos::parameterList();
        bad_verb->sublist("VerboseObject").set<std::string>("Verbosity Level", "loud");
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterValue>(
            [&] { f.setParameterList(bad_verb); }));
        EXPECT(f.getParameterList().is_null());  // failed lists are not kept
        EXPECT(throws<MCLS::Assertion>([&] { f.setParameterList(Teuchos::null); }));
    }

    g_section = "solver type -> manager";
    {
        struct Case {
            const char* type;
            const char* description;
        };
        const Case cases[] = {{"MCSA", "Adjoint MCSA (GPU)"},
                              {"Adjoint MC", "Adjoint MC (GPU)"},
                              {"Forward MC", "Forward MC (GPU)"},
                              {"Fixed Point", "Fixed Point (GPU)"},
                              {"Anderson", "Adjoint Anderson (GPU)"},
                              {"Adjoint MCSA", "Adjoint MCSA (GPU)"},
                              {"Forward MCSA", "Forward MCSA (GPU)"},
                              {"Adjoint Anderson", "Adjoint Anderson (GPU)"},
                              {"Forward Anderson", "Forward Anderson (GPU)"}};
        for (const Case& c : cases) {
            g_section = std::string("solver type ") + c.type;
            Factory f;
            auto pl = Teuchos::parameterList();
            pl->set<std::string>("Solver Type", c.type);
            f.setParameterList(pl);
            auto op = f.createOp();
            EXPECT(!op->isInitialized());
            f.initializeOp(A, op.get());
            EXPECT(op->isInitialized() && op->dim() == n);
            auto solver = op->solver()->getSolver();
            EXPECT(solver->description() == c.description);
            // The manager reads the factory's sublist itself, not a copy.
            EXPECT(op->solver()->getCurrentParameters().get() ==
                   &pl->sublist("Solver Types").sublist(c.type));
            EXPECT(op->description().find(c.description) != std::string::npos);
        }
        g_section = "solver type casts";
        Factory f;
        auto op = f.createOp();
        f.initializeOp(A, op.get());  // no parameter list: "MCSA" with an empty list
        EXPECT(Teuchos::nonnull(Teuchos::rcp_dynamic_cast<MCLS::MCSASolverManager<
                                    Vec, Mat, MCLS::AdjointTag>>(op->solver()->getSolver())));
        EXPECT(op->defaultTolerance() == 1.0);  // the MCSA manager's valid default
        auto pl = Teuchos::parameterList();
        pl->set<std::string>("Solver Type", "Forward MC");
        f.setParameterList(pl);
        f.initializeOp(A, op.get());
        EXPECT(Teuchos::nonnull(Teuchos::rcp_dynamic_cast<MCLS::MonteCarloSolverManager<
                                    Vec, Mat, MCLS::ForwardTag>>(op->solver()->getSolver())));
        EXPECT(op->defaultTolerance() == MCLS::SolveCriteria::unspecifiedTolerance());
        pl->set<std::string>("Solver Type", "Fixed Point");
        pl->sublist("Solver Types").sublist("Fixed Point").set<double>("Convergence Tolerance",
                                                                       1.0e-9);
        f.setParameterList(pl);
        f.initializeOp(A, op.get());
        EXPECT(op->defaultTolerance() == 1.0e-9);
        // An invalid manager setting surfaces when the manager is created.
        pl->set<std::string>("Solver Type", "Anderson");
        pl->sublist("Solver Types").sublist("Anderson").sublist("Anderson Parameters").set<int>(
            "Storage Depth", 40);
        f.setParameterList(pl);
        EXPECT(throws<MCLS::Assertion>([&] { f.initializeOp(A, op.get()); }));
    }

    g_section = "solve supports";
    {
        Factory f;
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        EXPECT(op->solveSupports(MCLS::NOTRANS));
        EXPECT(!op->solveSupports(MCLS::TRANS) && !op->solveSupports(MCLS::CONJTRANS));
        MCLS::SolveCriteria c(MCLS::SolveMeasureType(MCLS::SOLVE_MEASURE_NORM_RESIDUAL,
                                                     MCLS::SOLVE_MEASURE_NORM_RHS),
                              1e-6);
        EXPECT(op->solveSupports(MCLS::NOTRANS, &c));
        EXPECT(!op->solveSupportsSolveMeasureType(
            MCLS::NOTRANS, MCLS::SolveMeasureType(MCLS::SOLVE_MEASURE_NORM_RESIDUAL,
                                                  MCLS::SOLVE_MEASURE_NORM_INIT_RESIDUAL)));
        EXPECT(op->solveSupportsSolveMeasureType(MCLS::NOTRANS, MCLS::SolveMeasureType()));
        EXPECT(op->opSupported(MCLS::NOTRANS) && !op->opSupported(MCLS::TRANS));
    }

    g_section = "column loop over a host solver";
    {
        auto spl = Teuchos::parameterList();
        spl->set<double>("Convergence Tolerance", 1.0e-10);
        Teuchos::RCP<HostJacobi> jac;
        auto op = host_lows(A, spl, &jac);
        EXPECT(op->defaultTolerance() == 1.0e-10);
        MV B = block(n, {-1.0, 2.0, 0.5, -3.0});
        B[2][4] = 7.0;
        MV X = block(n, {0.0, 0.0, 0.0, 0.0});
        X[1][0] = 1.0;  // an initial guess is kept as the start
        auto st = op->solve(MCLS::NOTRANS, B, &X);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED);
        EXPECT(jac->tolerances.size() == 4);
        for (double t : jac->tolerances) EXPECT(t == 1.0e-10);
        int total = 0;
        double worst = 0.0;
        for (int j = 0; j < 4; ++j) {
            const double r = rel_residual(*A, X[j], B[j]);
            worst = std::max(worst, r);
            EXPECT(r <= 1.0e-10);
            EXPECT(rel_err(X[j], direct(*A, B[j])) < 1e-9);
        }
        total = st.extraParameters->get<int>("Iteration Count");
        EXPECT(total == st.extraParameters->get<int>("MCLS/Iteration Count") && total > 4);
        EXPECT(st.achievedTol == worst &&
               st.extraParameters->get<double>("MCLS/Achieved Tolerance") == worst);
        EXPECT(st.message.find("\"host Jacobi\"") != std::string::npos);
        EXPECT(st.message.find("SOLVE_STATUS_CONVERGED") != std::string::npos);
        EXPECT(st.message.find("for 4 RHSs using " + std::to_string(total)) != std::string::npos);
        // X and B are not held after the solve.
        EXPECT(op->problem()->getLHS().is_null() && op->problem()->getRHS().is_null());
        // The solver keeps the solve's copy of its parameters, not the original.
        EXPECT(jac->getCurrentParameters().get() != spl.get() &&
               !spl->isParameter("Maximum Iterations"));

        g_section = "requested tolerance and iteration limit";
        MV X2 = block(n, {0.0, 0.0});
        MV B2 = block(n, {1.0, -1.0});
        auto extra = Teuchos::parameterList();
        extra->set<int>("Maximum Iterations", 3);
        MCLS::SolveCriteria crit(MCLS::SolveMeasureType(MCLS::SOLVE_MEASURE_NORM_RESIDUAL,
                                                        MCLS::SOLVE_MEASURE_NORM_RHS),
                                 1.0e-12, extra);
        st = op->solve(MCLS::NOTRANS, B2, &X2, &crit);
        EXPECT(jac->tolerances.back() == 1.0e-12 && jac->limits.back() == 3);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_UNCONVERGED);
        EXPECT(st.extraParameters->get<int>("Iteration Count") == 6);
        EXPECT(st.achievedTol > 1.0e-12);
        // The default measure ignores a requested tolerance (as the
        // reference does); an unspecified one keeps the default.
        MCLS::SolveCriteria dflt(MCLS::SolveMeasureType(), 1.0e-3);
        X2 = block(n, {0.0});
        B2 = block(n, {1.0});
        op->solve(MCLS::NOTRANS, B2, &X2, &dflt);
        EXPECT(jac->tolerances.back() == 1.0e-10 && jac->limits.back() == 3);
        MCLS::SolveCriteria unspec(MCLS::SolveMeasureType(MCLS::SOLVE_MEASURE_NORM_RESIDUAL,
                                                          MCLS::SOLVE_MEASURE_NORM_RHS),
                                   MCLS::SolveCriteria::unspecifiedTolerance());
        X2 = block(n, {0.0});
        op->solve(MCLS::NOTRANS, B2, &X2, &unspec);
        EXPECT(jac->tolerances.back() == 1.0e-10);

        g_section = "block edge cases";
        MV empty_x, empty_b;
        const size_t before = jac->tolerances.size();
        st = op->solve(MCLS::NOTRANS, empty_b, &empty_x);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED && st.achievedTol == 0.0);
        EXPECT(st.extraParameters->get<int>("Iteration Count") == 0);
        EXPECT(jac->tolerances.size() == before);
        MV X3 = block(n, {0.0, 0.0});
        MV B3 = block(n, {1.0});
        EXPECT(throws<MCLS::Assertion>([&] { op->solve(MCLS::NOTRANS, B3, &X3); }, "column"));
        EXPECT(op->problem()->getLHS().is_null());
        EXPECT(throws<MCLS::Assertion>([&] { op->solve(MCLS::TRANS, B3, &X3); },
                                       "Solve does not support transpose type."));
        MCLS::SolveCriteria init(MCLS::SolveMeasureType(MCLS::SOLVE_MEASURE_NORM_RESIDUAL,
                                                        MCLS::SOLVE_MEASURE_NORM_INIT_RESIDUAL),
                                 1e-6);
        EXPECT(throws<MCLS::Assertion>([&] { op->solve(MCLS::NOTRANS, B3, &X3, &init); }));
        EXPECT(throws<MCLS::Assertion>([&] { op->solve(MCLS::NOTRANS, B3, nullptr); }));
        Lows blank;
        EXPECT(throws<MCLS::Assertion>([&] { blank.solve(MCLS::NOTRANS, B3, &X3); }));
    }

    g_section = "apply";
    {
        Teuchos::RCP<HostJacobi> jac;
        auto op = host_lows(A, Teuchos::parameterList(), &jac);
        EXPECT(op->defaultTolerance() == 1.0e-6);  // HostJacobi's valid default
        MV X = block(n, {1.0, -2.0});
        X[0][3] = 5.0;
        MV Y = block(n, {1.0, 1.0});
        op->apply(MCLS::NOTRANS, X, &Y, 2.0, 0.5);
        for (int j = 0; j < 2; ++j) {
            Vec ax;
            MCLS::MatrixTraits<Vec, Mat>::apply(*A, X[j], ax);
            for (int i = 0; i < n; ++i) EXPECT(std::fabs(Y[j][i] - (2.0 * ax[i] + 0.5)) < 1e-15);
        }
        MV Z = block(n, {std::nan("")});
        MV X1 = block(n, {1.0});
        op->apply(MCLS::NOTRANS, X1, &Z);  // beta = 0 overwrites, NaN included
        for (double z : Z[0]) EXPECT(std::isfinite(z));
        EXPECT(throws<MCLS::Assertion>([&] { op->apply(MCLS::TRANS, X1, &Z); }));
        EXPECT(throws<MCLS::Assertion>([&] { op->apply(MCLS::NOTRANS, X, &Z); }));
    }

    g_section = "preconditioner factory (host preconditioner)";
    {
        auto pf = Teuchos::rcp(new CountingPrecFactory());
        Factory f(pf);
        EXPECT(f.getPreconditionerFactory() == pf);
        EXPECT(f.supportsPreconditionerInputType(MCLS::PRECONDITIONER_INPUT_TYPE_AS_MATRIX));
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        EXPECT(pf->created == 1 && pf->built == 1 && pf->last_operator == A.get());
        EXPECT(Teuchos::nonnull(op->prec()) && !op->isExternalPrec());
        EXPECT(Teuchos::nonnull(op->problem()->getLeftPrec()) &&
               op->problem()->getRightPrec().is_null());
        auto kept = op->prec();
        f.initializeAndReuseOp(A, op.get());  // same preconditioner, not rebuilt
        EXPECT(pf->created == 1 && pf->built == 1 && op->prec() == kept);
        f.initializeOp(A, op.get());  // same object, rebuilt
        EXPECT(pf->created == 1 && pf->built == 2 && op->prec() == kept);
        auto approx = tridiag(n);
        f.initializeApproxPreconditionedOp(A, approx, op.get());
        EXPECT(pf->built == 3 && pf->last_operator == approx.get());
        EXPECT(op->approxOp() == approx && op->problem()->getOperator() == A);
        // A caller's preconditioner is used as given and handed back.
        auto mine = Teuchos::rcp(new HostDiagPrec());
        mine->setOperator(A);
        mine->buildPreconditioner();
        f.initializePreconditionedOp(A, mine, op.get());
        EXPECT(pf->built == 3 && op->isExternalPrec() && op->prec() == mine);
        EXPECT(op->problem()->getLeftPrec() == mine->getLeftPreconditioner());
        Teuchos::RCP<const Mat> A_out;
        Teuchos::RCP<MCLS::Preconditioner<Mat>> P_out;
        f.uninitializeOp(op.get(), &A_out, &P_out);
        EXPECT(A_out == A && P_out == mine && !op->isInitialized());
        // Matrices built elsewhere, right side only.
        auto PR = mine->getLeftPreconditioner();
        f.initializePreconditionedOp(A, Teuchos::null, PR, op.get());
        EXPECT(op->isExternalPrec() && op->problem()->getLeftPrec().is_null() &&
               op->problem()->getRightPrec() == PR && pf->built == 3);
        EXPECT(throws<MCLS::Assertion>([&] {
            f.initializePreconditionedOp(A, Teuchos::null, Teuchos::null, op.get());
        }));
        f.uninitializeOp(op.get());
        f.initializeOp(A, op.get());
        f.uninitializeOp(op.get(), &A_out, &P_out);
        EXPECT(P_out.is_null());  // the factory's own preconditioner is not handed out
        Teuchos::RCP<MCLS::PreconditionerFactoryBase<Mat>> out_f;
        std::string out_name;
        f.unsetPreconditionerFactory(&out_f, &out_name);
        EXPECT(out_f == pf && f.getPreconditionerFactory().is_null());

        // The subproblems carry the preconditioner to the manager.
        Teuchos::RCP<HostJacobi> jac;
        auto hop = host_lows(A, Teuchos::parameterList(), &jac, mine->getLeftPreconditioner());
        MV X = block(n, {0.0, 0.0});
        MV B = block(n, {1.0, 2.0});
        hop->solve(MCLS::NOTRANS, B, &X);
        EXPECT(jac->with_left.size() == 2 && jac->with_left[0] && jac->with_left[1]);
    }

    g_section = "GPU preconditioner factory";
    {
        MCLS::PreconditionerFactory<Vec, Mat> pf;
        auto v = pf.getValidParameters();
        EXPECT(v->get<std::string>("Preconditioner Type") == "Point Jacobi");
        EXPECT(v->sublist("Preconditioner Types").sublist("Block Jacobi").get<int>(
                   "Jacobi Block Size") == 1);
        auto pl = Teuchos::parameterList();
        pl->set<std::string>("Preconditioner Type", "Block Jacobi");
        pl->sublist("Preconditioner Types").sublist("Block Jacobi").set<int>("Jacobi Block Size",
                                                                             2);
        pl->sublist("Preconditioner Types").sublist("ILUT").set<double>("fact: drop tolerance",
                                                                        1e-2);
        pf.setParameterList(pl);
        EXPECT(pf.precType() == "Block Jacobi");
        auto p = pf.createPrec();
        EXPECT(Teuchos::nonnull(
            Teuchos::rcp_dynamic_cast<MCLS::BlockJacobiPreconditioner<Vec, Mat>>(p)));
        EXPECT(p->getCurrentParameters().get() ==
               &pl->sublist("Preconditioner Types").sublist("Block Jacobi"));
        for (const char* t : {"ILUT", "ParaSails", "PSILUT", "ML"}) {
            pl->set<std::string>("Preconditioner Type", t);
            pf.setParameterList(pl);
            EXPECT(throws<MCLS::Assertion>([&] { pf.createPrec(); }, t));
        }
        pl->set<std::string>("Preconditioner Type", "Amesos");
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterValue>(
            [&] { pf.setParameterList(pl); }));
        pl->set<std::string>("Preconditioner Type", "Point Jacobi");
        pf.setParameterList(pl);
        // Building needs the device: reported through MCLS::Assertion.
        auto pj = pf.createPrec();
        EXPECT(throws<MCLS::Assertion>([&] { pf.initializePrec(A, pj.get()); },
                                       "no usable CUDA device"));
        EXPECT(pf.isCompatible(*A));
    }

    g_section = "GPU manager without a device";
    {
        Factory f;
        auto pl = Teuchos::parameterList();
        pl->sublist("Solver Types").sublist("MCSA").set<bool>("Print Iterations", false);
        f.setParameterList(pl);
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        MV X = block(n, {0.0});
        MV B = block(n, {-1.0});
        EXPECT(throws<MCLS::Assertion>([&] { op->solve(MCLS::NOTRANS, B, &X); },
                                       "no usable CUDA device"));
        EXPECT(op->problem()->getLHS().is_null() && op->problem()->getRHS().is_null());
    }

    g_section = "verbose output";
    {
        const std::string file = dir + "/lows_verbose.txt";
        Factory f;
        auto pl = Teuchos::parameterList();
        PL& vo = pl->sublist("VerboseObject");
        vo.set<std::string>("Verbosity Level", "medium");
        vo.set<std::string>("Output File", file);
        f.setParameterList(pl);
        EXPECT(f.getVerbLevel() == MCLS::VERB_MEDIUM);
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        EXPECT(op->getVerbLevel() == MCLS::VERB_MEDIUM);
        std::ostringstream os;
        Teuchos::RCP<HostJacobi> jac;
        auto hop = host_lows(A, Teuchos::parameterList(), &jac);
        hop->setOStream(&os);
        hop->setVerbLevel(MCLS::VERB_LOW);
        MV X = block(n, {0.0});
        MV B = block(n, {1.0});
        hop->solve(MCLS::NOTRANS, B, &X);
        EXPECT(os.str().find("Solving block system using MCLS") != std::string::npos);
        EXPECT(os.str().find("Total solve time = ") != std::string::npos);
        std::ifstream in(file);
        std::stringstream text;
        text << in.rdbuf();
        EXPECT(text.str().find("Entering MCLS::LinearOpWithSolveFactory::initializeOp") !=
               std::string::npos);
        auto bad = Teuchos::parameterList();
        bad->sublist("VerboseObject").set<std::string>("Output File", dir + "/no/such/dir/x");
        EXPECT(throws<Teuchos::Exceptions::InvalidParameterValue>(
            [&] { f.setParameterList(bad); }));
    }
}

// The MCSA settings of the reference's manager tests, in `types`'s sublist `name`.
static void mcsa_sublist(PL& types, const char* name) {
    PL& s = types.sublist(name);
    s.set<double>("Convergence Tolerance", 1.0e-8);
    s.set<int>("Maximum Iterations", 20);
    s.set<int>("MC Check Frequency", 50);
    s.set<double>("Sample Ratio", 1.0);
    s.set<std::string>("Transport Type", "Global");
    s.set<bool>("Print Iterations", false);
}

static void gpu_checks() {
    const int n = 10;
    auto A = tridiag(n);

    // MCSA over a block of three right-hand sides; one manager and one
    // device domain serve every column.
    {
        g_section = "MCSA block solve";
        Factory f;
        auto pl = Teuchos::parameterList();
        mcsa_sublist(pl->sublist("Solver Types"), "MCSA");
        f.setParameterList(pl);
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        EXPECT(op->defaultTolerance() == 1.0e-8);
        MV B = block(n, {-1.0, 2.0, -2.0});
        MV X = block(n, {0.0, 0.0, 0.0});
        auto st = op->solve(MCLS::NOTRANS, B, &X);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED);
        EXPECT(st.achievedTol > 0.0 && st.achievedTol <= 1.0e-8);
        const int its = st.extraParameters->get<int>("Iteration Count");
        EXPECT(its >= 3 && its < 60);
        for (int j = 0; j < 3; ++j) {
            for (double xi : X[j]) EXPECT(B[j][0] < 0 ? xi < 0.0 : xi > 0.0);
            EXPECT(rel_err(X[j], direct(*A, B[j])) < 1e-7);
            EXPECT(rel_residual(*A, X[j], B[j]) < 2.0e-8);
        }
        // A second block on the same op continues with the same manager.
        MV B2 = block(n, {1.0});
        MV X2 = block(n, {0.0});
        st = op->solve(MCLS::NOTRANS, B2, &X2);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED);
        EXPECT(rel_err(X2[0], direct(*A, B2[0])) < 1e-7);
    }

    // "Fixed Point" (Richardson): the reference's 15 iterations per
    // right-hand side, with the tolerance coming from the solve criteria.
    {
        g_section = "Fixed Point block solve";
        auto F = fixed_point_matrix(n);
        Factory f;
        auto pl = Teuchos::parameterList();
        pl->set<std::string>("Solver Type", "Fixed Point");
        PL& fp = pl->sublist("Solver Types").sublist("Fixed Point");
        fp.set<double>("Convergence Tolerance", 1.0);
        fp.set<int>("Maximum Iterations", 100);
        fp.set<double>("Richardson Relaxation", 1.0);
        fp.set<bool>("Print Iterations", false);
        f.setParameterList(pl);
        auto op = f.createOp();
        f.initializeOp(F, op.get());
        MV B = block(n, {-1.0, 2.0});
        MV X = block(n, {0.0, 0.0});
        MCLS::SolveCriteria crit(MCLS::SolveMeasureType(MCLS::SOLVE_MEASURE_NORM_RESIDUAL,
                                                        MCLS::SOLVE_MEASURE_NORM_RHS),
                                 1.0e-8);
        auto st = op->solve(MCLS::NOTRANS, B, &X, &crit);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED);
        EXPECT(st.extraParameters->get<int>("Iteration Count") == 30);
        for (int j = 0; j < 2; ++j)
            for (double xi : X[j]) EXPECT(B[j][0] < 0 ? xi < 0.0 : xi > 0.0);
    }

    // The "Point Jacobi" preconditioner factory: built on the device and
    // handed to the MCSA manager.
    {
        g_section = "Point Jacobi preconditioner factory";
        auto pf = Teuchos::rcp(new MCLS::PreconditionerFactory<Vec, Mat>());
        auto ppl = Teuchos::parameterList();
        ppl->set<std::string>("Preconditioner Type", "Point Jacobi");
        pf->setParameterList(ppl);
        Factory f(pf);
        auto pl = Teuchos::parameterList();
        mcsa_sublist(pl->sublist("Solver Types"), "MCSA");
        f.setParameterList(pl);
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        auto PL_ = op->problem()->getLeftPrec();
        EXPECT(Teuchos::nonnull(PL_) && PL_->n == n && PL_->values.size() == size_t(n));
        MV B = block(n, {2.0, -1.0});
        MV X = block(n, {0.0, 0.0});
        auto st = op->solve(MCLS::NOTRANS, B, &X);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED);
        for (int j = 0; j < 2; ++j) EXPECT(rel_err(X[j], direct(*A, B[j])) < 1e-7);
    }

    // "Anderson": Anderson-accelerated MCSA behind the same interface.
    {
        g_section = "Anderson block solve";
        Factory f;
        auto pl = Teuchos::parameterList();
        pl->set<std::string>("Solver Type", "Anderson");
        mcsa_sublist(pl->sublist("Solver Types"), "Anderson");
        PL& a = pl->sublist("Solver Types").sublist("Anderson");
        a.set<int>("Maximum Iterations", 100);
        a.set<double>("Sample Ratio", 10.0);
        a.sublist("Anderson Parameters").set<int>("Storage Depth", 3);
        f.setParameterList(pl);
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        MV B = block(n, {-1.0, 2.0});
        MV X = block(n, {0.0, 0.0});
        auto st = op->solve(MCLS::NOTRANS, B, &X);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED);
        EXPECT(st.achievedTol < 1.0e-8);
        for (int j = 0; j < 2; ++j) EXPECT(rel_err(X[j], direct(*A, B[j])) < 1e-7);
    }
}

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    const std::string dir = argc > 2 ? argv[2] : ".";
    try {
        if (gpu) gpu_checks();
        else cpu_checks(dir);
    } catch (const std::exception& e) {
        std::printf("FAILED in %s: exception %s\n", g_section.c_str(), e.what());
        return 2;
    }
    std::printf("%s: %d failure(s)\n", gpu ? "gpu" : "cpu", g_failures);
    return g_failures ? 1 : 0;
}
