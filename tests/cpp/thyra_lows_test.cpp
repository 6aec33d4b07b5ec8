// Thyra layer test: include/Thyra_MCLSGpuLinearOpWithSolveFactory.hpp
// compiled against the stand-ins of Thyra's and Tpetra's interfaces
// (tests/cpp/thyra_standin, tests/cpp/tpetra_standin; no Trilinos here).
//
//   thyra_lows_test cpu   the factory's parameters, compatibility, solve
//                         support, apply, preconditioned ops and
//                         uninitializeOp; the solve's translation of Thyra
//                         criteria and statuses over a host solver; a GPU
//                         solve without a device throws MCLS::Assertion.
//   thyra_lows_test gpu   blocks of right-hand sides solved on the device
//                         through the Thyra interface ("MCSA", with and
//                         without a Thyra preconditioner).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "Thyra_MCLSGpuLinearOpWithSolveFactory.hpp"

typedef Tpetra::Map<int, long long> TMap;
typedef Tpetra::Vector<double, int, long long> TV;
typedef Tpetra::MultiVector<double, int, long long> TMV;
typedef Tpetra::CrsMatrix<double, int, long long> TM;
typedef Tpetra::DefaultNode Node;
typedef Thyra::MCLSGpuLinearOpWithSolveFactory<int, long long, Node> Factory;
typedef Thyra::MCLSGpuLinearOpWithSolve<int, long long, Node> Lows;
typedef MCLS::VectorTraits<TV> VT;
typedef MCLS::MatrixTraits<TV, TM> MT;

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

template <class F>
static bool throws_assertion(F&& f, const char* needle) {
    try {
        f();
    } catch (const MCLS::Assertion& e) {
        return std::string(e.what()).find(needle) != std::string::npos;
    }
    return false;
}

static Teuchos::RCP<TM> tridiag(int n) {
    auto map = Teuchos::rcp(new TMap(std::size_t(n), 0, Tpetra::getDefaultComm()));
    auto A = Teuchos::rcp(new TM(map, 3));
    for (int i = 0; i < n; ++i) {
        const int c0 = i == 0 ? 0 : (i == n - 1 ? n - 3 : i - 1);
        for (int c = c0; c < c0 + 3; ++c) {
            const double v = c == i ? 1.0 : (std::abs(c - i) == 1 ? -0.14 : 0.0);
            const long long g = c;
            A->insertGlobalValues(i, 1, &v, &g);
        }
    }
    A->fillComplete();
    return A;
}

static Teuchos::RCP<TM> scaled_identity(int n, double d) {
    auto map = Teuchos::rcp(new TMap(std::size_t(n), 0, Tpetra::getDefaultComm()));
    auto I = Teuchos::rcp(new TM(map, 1));
    for (int i = 0; i < n; ++i) {
        const long long g = i;
        I->insertGlobalValues(i, 1, &d, &g);
    }
    I->fillComplete();
    return I;
}

static Teuchos::RCP<const Thyra::LinearOpBase<double>> thyra_op(const Teuchos::RCP<TM>& A) {
    return Thyra::createConstLinearOp<double, int, long long, Node>(
        Teuchos::RCP<const Tpetra::Operator<double, int, long long, Node>>(A));
}

static std::vector<double> direct(const TM& A, std::vector<double> b) {
    std::vector<std::int64_t> rp, ci;
    std::vector<double> v;
    MT::getCsr(A, rp, ci, v);
    const int n = int(b.size());
    std::vector<double> M(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (auto p = rp[i]; p < rp[i + 1]; ++p) M[size_t(i) * n + ci[p]] += v[p];
    for (int k = 0; k < n; ++k)
        for (int i = k + 1; i < n; ++i) {
            const double f = M[size_t(i) * n + k] / M[size_t(k) * n + k];
            for (int j = k; j < n; ++j) M[size_t(i) * n + j] -= f * M[size_t(k) * n + j];
            b[i] -= f * b[k];
        }
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) b[i] -= M[size_t(i) * n + j] * b[j];
        b[i] /= M[size_t(i) * n + i];
    }
    return b;
}

// Host Jacobi behind the SolverManager interface: records the tolerance and
// iteration limit each solve was given.
class HostJacobi : public MCLS::SolverManager<TV, TM> {
  public:
    typedef MCLS::LinearProblem<TV, TM> LP;
    explicit HostJacobi(const Teuchos::RCP<Teuchos::ParameterList>& pl) : d_pl(pl) {}
    const LP& getProblem() const override { return *d_lp; }
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<double>("Convergence Tolerance", 1e-10);
        return pl;
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return d_pl;
    }
    double achievedTol() const override { return d_res; }
    int getNumIters() const override { return d_iters; }
    void setProblem(const Teuchos::RCP<LP>& p) override { d_lp = p; }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& p) override { d_pl = p; }
    bool solve() override {
        tol = d_pl->get<double>("Convergence Tolerance");
        maxit = d_pl->isParameter("Maximum Iterations") ? d_pl->get<int>("Maximum Iterations") : 500;
        const std::int64_t n = VT::getGlobalLength(*d_lp->getRHS());
        double bn = 0.0;
        for (std::int64_t i = 0; i < n; ++i) bn += std::pow(VT::view(*d_lp->getRHS())[i], 2);
        d_iters = 0;
        for (;;) {
            d_lp->updateResidual();
            const double* r = VT::view(*d_lp->getResidual());
            double rn = 0.0;
            for (std::int64_t i = 0; i < n; ++i) rn += r[i] * r[i];
            d_res = std::sqrt(rn / bn);
            if (d_res <= tol || d_iters >= maxit) break;
            auto upd = VT::clone(*d_lp->getLHS());
            for (std::int64_t i = 0; i < n; ++i) VT::viewNonConst(*upd)[i] = r[i];  // diag = 1
            d_lp->updateSolution(upd);
            ++d_iters;
        }
        return d_res <= tol;
    }
    bool getConvergedStatus() const override { return d_res <= tol; }
    std::string description() const override { return "host Jacobi"; }
    double tol = 0.0;
    int maxit = 0;

  private:
    Teuchos::RCP<Teuchos::ParameterList> d_pl;
    Teuchos::RCP<LP> d_lp;
    double d_res = 0.0;
    int d_iters = 0;
};

// An operator that is not a CRS matrix.
class OtherOp : public Tpetra::Operator<double, int, long long, Node> {};

static void cpu_checks() {
    const int n = 10;
    auto A = tridiag(n);
    auto src = Thyra::defaultLinearOpSource<double>(thyra_op(A));

    g_section = "factory";
    Factory f;
    EXPECT(f.getValidParameters()->get<std::string>("Solver Type") == "MCSA");
    EXPECT(f.description() == "Thyra::MCLSGpuLinearOpWithSolveFactory");
    auto pl = Teuchos::parameterList();
    pl->sublist("Solver Types").sublist("MCSA").set<bool>("Print Iterations", false);
    f.setParameterList(pl);
    EXPECT(f.getParameterList() == pl && f.getNonconstParameterList() == pl);
    EXPECT(f.isCompatible(*src));
    auto other = Thyra::defaultLinearOpSource<double>(Thyra::createConstLinearOp<double, int, long long, Node>(
        Teuchos::RCP<const Tpetra::Operator<double, int, long long, Node>>(Teuchos::rcp(new OtherOp()))));
    EXPECT(!f.isCompatible(*other));
    EXPECT(f.supportsPreconditionerInputType(Thyra::PRECONDITIONER_INPUT_TYPE_AS_OPERATOR));

    g_section = "initializeOp and solve support";
    auto op = f.createOp();
    f.initializeOp(src, op.get());
    EXPECT(op->range()->dim() == n && op->domain()->dim() == n);
    EXPECT(op->solveSupports(Thyra::NOTRANS) && !op->solveSupports(Thyra::TRANS));
    Thyra::SolveCriteria<double> rr(
        Thyra::SolveMeasureType(Thyra::SOLVE_MEASURE_NORM_RESIDUAL, Thyra::SOLVE_MEASURE_NORM_RHS),
        1e-6);
    EXPECT(op->solveSupports(Thyra::NOTRANS, Teuchos::ptr(&rr)));
    EXPECT(!op->solveSupportsSolveMeasureType(
        Thyra::NOTRANS, Thyra::SolveMeasureType(Thyra::SOLVE_MEASURE_NORM_RESIDUAL,
                                                Thyra::SOLVE_MEASURE_NORM_INIT_RESIDUAL)));
    EXPECT(op->opSupported(Thyra::NOTRANS) && !op->opSupported(Thyra::TRANS));
    EXPECT(throws_assertion([&] { f.initializeOp(other, op.get()); }, "not a Tpetra::CrsMatrix"));

    g_section = "apply";
    auto X = Teuchos::rcp(new TMV(A->getRowMap(), 2));
    auto Y = Teuchos::rcp(new TMV(A->getRowMap(), 2));
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < n; ++i) X->at(i, j) = 1.0 + i + 10 * j;
    auto Xt = Thyra::createMultiVector<double, int, long long, Node>(X);
    auto Yt = Thyra::createMultiVector<double, int, long long, Node>(Y);
    op->apply(Thyra::NOTRANS, *Xt, Teuchos::ptr(Yt.get()), 2.0, 0.0);
    TMV AX(A->getRowMap(), 2);
    A->apply(*X, AX);
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < n; ++i) EXPECT(std::fabs(Y->at(i, j) - 2.0 * AX.at(i, j)) < 1e-14);

    g_section = "solve without a device";
    auto B = Teuchos::rcp(new TMV(A->getRowMap(), 1));
    auto Bt = Thyra::createMultiVector<double, int, long long, Node>(B);
    auto X1t = Thyra::createMultiVector<double, int, long long, Node>(
        Teuchos::rcp(new TMV(A->getRowMap(), 1)));
    EXPECT(throws_assertion([&] { op->solve(Thyra::NOTRANS, *Bt, Teuchos::ptr(X1t.get())); },
                            "no usable CUDA device"));
    EXPECT(throws_assertion([&] { op->solve(Thyra::NOTRANS, *Bt, Teuchos::ptr(Xt.get())); },
                            "column counts"));

    g_section = "criteria and status translation";
    {
        Lows& lows = Teuchos::dyn_cast<Lows>(*op);
        auto spl = Teuchos::parameterList();
        spl->set<double>("Convergence Tolerance", 1e-10);
        auto jac = Teuchos::rcp(new HostJacobi(spl));
        auto lp = Teuchos::rcp(new MCLS::LinearProblemAdapter<TMV, TM>());
        lp->setOperator(A);
        auto adapter = Teuchos::rcp(new MCLS::SolverManagerAdapter<TMV, TM>(jac));
        adapter->setProblem(lp);
        lows.core().initialize(lp, spl, adapter);
        auto B2 = Teuchos::rcp(new TMV(A->getRowMap(), 2));
        auto X2 = Teuchos::rcp(new TMV(A->getRowMap(), 2));
        for (int i = 0; i < n; ++i) {
            B2->at(i, 0) = -1.0;
            B2->at(i, 1) = 2.0;
        }
        auto B2t = Thyra::createMultiVector<double, int, long long, Node>(B2);
        auto X2t = Thyra::createMultiVector<double, int, long long, Node>(X2);
        auto st = op->solve(Thyra::NOTRANS, *B2t, Teuchos::ptr(X2t.get()));
        EXPECT(st.solveStatus == Thyra::SOLVE_STATUS_CONVERGED && st.achievedTol <= 1e-10);
        EXPECT(jac->tol == 1e-10);
        EXPECT(st.extraParameters->get<int>("Iteration Count") > 2);
        EXPECT(st.message.find("\"host Jacobi\"") != std::string::npos);
        for (int j = 0; j < 2; ++j) {
            const auto xs = direct(*A, std::vector<double>(size_t(n), j ? 2.0 : -1.0));
            for (int i = 0; i < n; ++i) EXPECT(std::fabs(X2->at(i, j) - xs[i]) < 1e-9);
        }
        auto extra = Teuchos::parameterList();
        extra->set<int>("Maximum Iterations", 2);
        Thyra::SolveCriteria<double> crit(
            Thyra::SolveMeasureType(Thyra::SOLVE_MEASURE_NORM_RESIDUAL, Thyra::SOLVE_MEASURE_NORM_RHS),
            1e-12, extra);
        for (int i = 0; i < n; ++i) X2->at(i, 0) = X2->at(i, 1) = 0.0;
        st = op->solve(Thyra::NOTRANS, *B2t, Teuchos::ptr(X2t.get()), Teuchos::ptr(&crit));
        EXPECT(jac->tol == 1e-12 && jac->maxit == 2);
        EXPECT(st.solveStatus == Thyra::SOLVE_STATUS_UNCONVERGED);
        EXPECT(st.extraParameters->get<int>("Iteration Count") == 4);
        Thyra::SolveCriteria<double> unspecified(
            Thyra::SolveMeasureType(Thyra::SOLVE_MEASURE_NORM_RESIDUAL, Thyra::SOLVE_MEASURE_NORM_RHS),
            Thyra::SolveCriteria<double>::unspecifiedTolerance());
        op->solve(Thyra::NOTRANS, *B2t, Teuchos::ptr(X2t.get()), Teuchos::ptr(&unspecified));
        EXPECT(jac->tol == 1e-10);
    }

    g_section = "preconditioned op and uninitializeOp";
    {
        auto PLm = scaled_identity(n, 1.0);
        auto prec = Teuchos::rcp(new Thyra::DefaultPreconditioner<double>(thyra_op(PLm), Teuchos::null));
        auto pop = f.createOp();
        f.initializePreconditionedOp(src, prec, pop.get());
        Lows& lows = Teuchos::dyn_cast<Lows>(*pop);
        EXPECT(lows.core().isExternalPrec());
        EXPECT(lows.core().problem()->getLeftPrec() == PLm &&
               lows.core().problem()->getRightPrec().is_null());
        Teuchos::RCP<const Thyra::LinearOpSourceBase<double>> src_out;
        Teuchos::RCP<const Thyra::PreconditionerBase<double>> prec_out;
        f.uninitializeOp(pop.get(), &src_out, &prec_out);
        EXPECT(src_out == src && prec_out == prec && !lows.core().isInitialized());
        EXPECT(throws_assertion([&] { f.initializePreconditionedOp(src, Teuchos::null, pop.get()); },
                                "null preconditioner"));
        f.initializeAndReuseOp(src, pop.get());
        EXPECT(lows.core().isInitialized());
    }
}

static void gpu_checks() {
    const int n = 10;
    auto A = tridiag(n);
    auto src = Thyra::defaultLinearOpSource<double>(thyra_op(A));
    for (int use_prec = 0; use_prec < 2; ++use_prec) {
        g_section = use_prec ? "MCSA through Thyra with a preconditioner" : "MCSA through Thyra";
        Factory f;
        auto pl = Teuchos::parameterList();
        auto& m = pl->sublist("Solver Types").sublist("MCSA");
        m.set<double>("Convergence Tolerance", 1.0e-8);
        m.set<int>("Maximum Iterations", 20);
        m.set<double>("Sample Ratio", 1.0);
        m.set<bool>("Print Iterations", false);
        f.setParameterList(pl);
        auto op = f.createOp();
        if (use_prec) {
            auto prec = Teuchos::rcp(new Thyra::DefaultPreconditioner<double>(
                thyra_op(scaled_identity(n, 1.0)), Teuchos::null));
            f.initializePreconditionedOp(src, prec, op.get());
        } else {
            f.initializeOp(src, op.get());
        }
        auto B = Teuchos::rcp(new TMV(A->getRowMap(), 2));
        auto X = Teuchos::rcp(new TMV(A->getRowMap(), 2));
        for (int i = 0; i < n; ++i) {
            B->at(i, 0) = -1.0;
            B->at(i, 1) = 2.0;
        }
        auto Bt = Thyra::createMultiVector<double, int, long long, Node>(B);
        auto Xt = Thyra::createMultiVector<double, int, long long, Node>(X);
        auto st = op->solve(Thyra::NOTRANS, *Bt, Teuchos::ptr(Xt.get()));
        EXPECT(st.solveStatus == Thyra::SOLVE_STATUS_CONVERGED);
        EXPECT(st.achievedTol > 0.0 && st.achievedTol <= 1e-8);
        for (int j = 0; j < 2; ++j) {
            const auto xs = direct(*A, std::vector<double>(size_t(n), j ? 2.0 : -1.0));
            double d = 0.0, s = 0.0;
            for (int i = 0; i < n; ++i) {
                d += std::pow(X->at(i, j) - xs[i], 2);
                s += xs[i] * xs[i];
            }
            EXPECT(std::sqrt(d / s) < 1e-7);
        }
    }
}

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    try {
        if (gpu) gpu_checks();
        else cpu_checks();
    } catch (const std::exception& e) {
        std::printf("FAILED in %s: exception %s\n", g_section.c_str(), e.what());
        return 2;
    }
    std::printf("%s: %d failure(s)\n", gpu ? "gpu" : "cpu", g_failures);
    return g_failures ? 1 : 0;
}
