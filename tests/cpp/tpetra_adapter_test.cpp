// Tpetra adapter test: include/MCLS_TpetraAdapter.hpp compiled against the
// stand-in of Tpetra's interface in tests/cpp/tpetra_standin (no Trilinos in
// this image).
//
//   tpetra_adapter_test cpu   the traits (CSR extraction from an unsorted,
//                             index-base-1 matrix, the round trip through
//                             fromCsr, y = A x, vector and multi-vector
//                             views), LinearProblem's host helpers on
//                             vectors that copy by view, a block solve over a
//                             multi-vector with a host solver, and the GPU
//                             managers instantiated on Tpetra types (a solve
//                             without a device throws MCLS::Assertion).
//   tpetra_adapter_test gpu   MCSA and a device-built point-Jacobi
//                             preconditioner on Tpetra types, after
//                             tpetra/test/tstTpetraMCSASolverManager.cpp:72-204.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "MCLS_TpetraAdapter.hpp"

typedef Tpetra::Map<int, long long> TMap;
typedef Tpetra::Vector<double, int, long long> TV;
typedef Tpetra::MultiVector<double, int, long long> TMV;
typedef Tpetra::CrsMatrix<double, int, long long> TM;
typedef MCLS::VectorTraits<TV> VT;
typedef MCLS::MatrixTraits<TV, TM> MT;
typedef MCLS::MultiVectorTraits<TMV, TM> MVT;

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

static Teuchos::RCP<const TMap> contiguous_map(int n, long long base) {
    return Teuchos::rcp(new TMap(std::size_t(n), base, Tpetra::getDefaultComm()));
}

// The reference's MCSA test matrix (1 on the diagonal, -0.14 beside it,
// explicit zeros closing the first and last rows), entries of each row
// inserted right to left, on global rows base .. base+n-1.
static Teuchos::RCP<TM> tridiag(int n, long long base = 0) {
    auto A = Teuchos::rcp(new TM(contiguous_map(n, base), 3));
    for (int i = 0; i < n; ++i) {
        const int c0 = i == 0 ? 0 : (i == n - 1 ? n - 3 : i - 1);
        for (int c = c0 + 2; c >= c0; --c) {
            const double v = c == i ? 1.0 : (std::abs(c - i) == 1 ? -0.14 : 0.0);
            const long long g = base + c;
            A->insertGlobalValues(base + i, 1, &v, &g);
        }
    }
    A->fillComplete();
    return A;
}

// Dense solve of the n x n CSR system.
static std::vector<double> direct(const std::vector<std::int64_t>& rp,
                                  const std::vector<std::int64_t>& ci,
                                  const std::vector<double>& v, std::vector<double> b) {
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

static void fill(TV& x, double v) {
    double* p = VT::viewNonConst(x);
    for (std::int64_t i = 0; i < VT::getGlobalLength(x); ++i) p[i] = v;
}

// Jacobi on the host behind the SolverManager interface, on Tpetra types.
class TpetraJacobi : public MCLS::SolverManager<TV, TM> {
  public:
    typedef MCLS::LinearProblem<TV, TM> LP;
    explicit TpetraJacobi(const Teuchos::RCP<Teuchos::ParameterList>& pl) : d_pl(pl) {}
    const LP& getProblem() const override { return *d_lp; }
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<double>("Convergence Tolerance", 1e-12);
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
        const double tol = d_pl->get<double>("Convergence Tolerance");
        std::vector<std::int64_t> rp, ci;
        std::vector<double> v;
        MT::getCsr(*d_lp->getOperator(), rp, ci, v);
        const std::int64_t n = std::int64_t(rp.size()) - 1;
        double bn = 0.0;
        const double* b = VT::view(*d_lp->getRHS());
        for (std::int64_t i = 0; i < n; ++i) bn += b[i] * b[i];
        bn = std::sqrt(bn);
        d_iters = 0;
        for (;;) {
            d_lp->updateResidual();
            const double* r = VT::view(*d_lp->getResidual());
            double rn = 0.0;
            for (std::int64_t i = 0; i < n; ++i) rn += r[i] * r[i];
            d_res = std::sqrt(rn) / bn;
            if (d_res <= tol || d_iters >= 500) break;
            auto upd = VT::clone(*d_lp->getLHS());
            double* u = VT::viewNonConst(*upd);
            for (std::int64_t i = 0; i < n; ++i)
                for (auto p = rp[i]; p < rp[i + 1]; ++p)
                    if (ci[p] == i) u[i] = r[i] / v[p];
            d_lp->updateSolution(upd);
            ++d_iters;
        }
        return d_res <= tol;
    }
    bool getConvergedStatus() const override { return d_res <= d_pl->get<double>("Convergence Tolerance"); }
    std::string description() const override { return "Tpetra host Jacobi"; }

  private:
    Teuchos::RCP<Teuchos::ParameterList> d_pl;
    Teuchos::RCP<LP> d_lp;
    double d_res = 0.0;
    int d_iters = 0;
};

static void cpu_checks() {
    const int n = 10;

    g_section = "CSR from an unsorted index-base-1 matrix";
    auto A1 = tridiag(n, 1);
    std::vector<std::int64_t> rp, ci;
    std::vector<double> v;
    MT::getCsr(*A1, rp, ci, v);
    EXPECT(MT::getGlobalNumRows(*A1) == n && rp.size() == size_t(n + 1) && rp[n] == 3 * n);
    for (int i = 0; i < n; ++i) {
        const int c0 = i == 0 ? 0 : (i == n - 1 ? n - 3 : i - 1);
        for (int k = 0; k < 3; ++k) {
            const auto p = rp[i] + k;
            EXPECT(ci[p] == c0 + k);
            const int c = c0 + k;
            EXPECT(v[p] == (c == i ? 1.0 : (std::abs(c - i) == 1 ? -0.14 : 0.0)));
        }
    }

    g_section = "maps the adapter rejects";
    {
        std::vector<long long> gids(n);
        for (int i = 0; i < n; ++i) gids[i] = n - 1 - i;
        auto pmap = Teuchos::rcp(new TMap(std::size_t(n), gids, 0, Tpetra::getDefaultComm()));
        auto P = Teuchos::rcp(new TM(pmap, 1));
        for (int i = 0; i < n; ++i) {
            const double one = 1.0;
            const long long g = i;
            P->insertGlobalValues(i, 1, &one, &g);
        }
        P->fillComplete();
        EXPECT(throws_assertion([&] { MT::getCsr(*P, rp, ci, v); }, "contiguous"));
        auto W = Teuchos::rcp(new TM(contiguous_map(n, 0), 1));
        const double one = 1.0;
        const long long outside = n + 3;
        W->insertGlobalValues(0, 1, &one, &outside);
        W->fillComplete();
        EXPECT(throws_assertion([&] { MT::getCsr(*W, rp, ci, v); }, "outside"));
    }

    g_section = "fromCsr round trip and y = A x";
    auto A = tridiag(n);
    MT::getCsr(*A, rp, ci, v);
    auto B = MT::fromCsr(n, rp, ci, v);
    std::vector<std::int64_t> rp2, ci2;
    std::vector<double> v2;
    MT::getCsr(*B, rp2, ci2, v2);
    EXPECT(rp2 == rp && ci2 == ci && v2 == v);
    TV x(A->getRowMap()), y(A->getRowMap());
    double* xp = VT::viewNonConst(x);
    for (int i = 0; i < n; ++i) xp[i] = 1.0 + i;
    MT::apply(*B, x, y);
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (auto p = rp[i]; p < rp[i + 1]; ++p) s += v[p] * (1.0 + ci[p]);
        EXPECT(std::fabs(VT::view(y)[i] - s) < 1e-15);
    }

    g_section = "vector and multi-vector views";
    {
        EXPECT(VT::getGlobalLength(x) == n);
        auto c = VT::clone(x);
        for (int i = 0; i < n; ++i) EXPECT(VT::view(*c)[i] == 0.0);
        TV alias = x;  // Tpetra copies by view
        VT::viewNonConst(alias)[2] = -7.0;
        EXPECT(VT::view(x)[2] == -7.0);
        TMV X(A->getRowMap(), 3);
        EXPECT(MVT::getNumVectors(X) == 3);
        VT::viewNonConst(*MVT::getVectorNonConst(X, 1))[4] = 2.5;
        EXPECT(X.at(4, 1) == 2.5 && MVT::getVector(X, 1)->getData()[4] == 2.5);
        EXPECT(X.at(4, 0) == 0.0 && X.at(4, 2) == 0.0);
    }

    g_section = "LinearProblem on vectors that copy by view";
    {
        auto xv = Teuchos::rcp(new TV(A->getRowMap()));
        auto bv = Teuchos::rcp(new TV(A->getRowMap()));
        fill(*xv, 2.0);
        fill(*bv, 5.0);
        MCLS::LinearProblem<TV, TM> lp(A, xv, bv);
        lp.setLeftPrec(B);
        lp.setRightPrec(B);
        TV out(A->getRowMap());
        lp.apply(*xv, out);  // B A B x, x untouched
        for (int i = 0; i < n; ++i) EXPECT(VT::view(*xv)[i] == 2.0);
        // Dense B A B x with B = A.
        std::vector<double> t(n, 2.0), u(n);
        for (int pass = 0; pass < 3; ++pass) {
            for (int i = 0; i < n; ++i) {
                double s = 0.0;
                for (auto p = rp[i]; p < rp[i + 1]; ++p) s += v[p] * t[ci[p]];
                u[i] = s;
            }
            t = u;
        }
        for (int i = 0; i < n; ++i) EXPECT(std::fabs(VT::view(out)[i] - t[i]) < 1e-14);
        lp.updatePrecResidual();
        std::vector<double> r(n);
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (auto p = rp[i]; p < rp[i + 1]; ++p) s += v[p] * 2.0;
            r[i] = 5.0 - s;
        }
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (auto p = rp[i]; p < rp[i + 1]; ++p) s += v[p] * r[ci[p]];
            EXPECT(std::fabs(VT::view(*lp.getPrecResidual())[i] - s) < 1e-14);
            EXPECT(std::fabs(VT::view(*lp.getResidual())[i] - r[i]) < 1e-14);
        }
        auto comp = lp.getCompositeOperator();
        EXPECT(MT::getGlobalNumRows(*comp) == n);
    }

    g_section = "block solve over a multi-vector";
    {
        auto spl = Teuchos::parameterList();
        spl->set<double>("Convergence Tolerance", 1e-12);
        auto solver = Teuchos::rcp(new TpetraJacobi(spl));
        auto lp = Teuchos::rcp(new MCLS::LinearProblemAdapter<TMV, TM>());
        lp->setOperator(A);
        auto adapter = Teuchos::rcp(new MCLS::SolverManagerAdapter<TMV, TM>(solver));
        adapter->setProblem(lp);
        MCLS::LinearOpWithSolve<TMV, TM> op;
        op.initialize(lp, spl, adapter);
        TMV Bm(A->getRowMap(), 3), Xm(A->getRowMap(), 3);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < n; ++i) Bm.at(i, j) = (j + 1) * (i % 2 ? 1.0 : -1.0);
        auto st = op.solve(MCLS::NOTRANS, Bm, &Xm);
        EXPECT(st.solveStatus == MCLS::SOLVE_STATUS_CONVERGED && st.achievedTol <= 1e-12);
        for (int j = 0; j < 3; ++j) {
            std::vector<double> bj(n);
            for (int i = 0; i < n; ++i) bj[i] = Bm.at(i, j);
            const auto xs = direct(rp, ci, v, bj);
            for (int i = 0; i < n; ++i) EXPECT(std::fabs(Xm.at(i, j) - xs[i]) < 1e-10);
        }
        TMV Ym(A->getRowMap(), 3);
        op.apply(MCLS::NOTRANS, Xm, &Ym);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < n; ++i) EXPECT(std::fabs(Ym.at(i, j) - Bm.at(i, j)) < 1e-11);
    }

    g_section = "GPU managers on Tpetra types";
    {
        MCLS::LinearOpWithSolveFactory<TMV, TM> f;
        auto pl = Teuchos::parameterList();
        pl->sublist("Solver Types").sublist("MCSA").set<bool>("Print Iterations", false);
        f.setParameterList(pl);
        auto op = f.createOp();
        f.initializeOp(A, op.get());
        TMV Bm(A->getRowMap(), 1), Xm(A->getRowMap(), 1);
        EXPECT(throws_assertion([&] { op->solve(MCLS::NOTRANS, Bm, &Xm); },
                                "no usable CUDA device"));
        MCLS::PointJacobiPreconditioner<TV, TM> prec;
        prec.setOperator(A);
        EXPECT(throws_assertion([&] { prec.buildPreconditioner(); }, "no usable CUDA device"));
    }
}

static void gpu_checks() {
    const int n = 10;
    auto A = tridiag(n, 1);  // index base 1: the adapter hands over 0-based CSR
    std::vector<std::int64_t> rp, ci;
    std::vector<double> v;
    MT::getCsr(*A, rp, ci, v);
    auto pl = Teuchos::parameterList();
    pl->set<double>("Convergence Tolerance", 1.0e-8);
    pl->set<int>("Maximum Iterations", 20);
    pl->set<double>("Sample Ratio", 1.0);
    pl->set<bool>("Print Iterations", false);
    for (int prec = 0; prec < 2; ++prec) {
        g_section = prec ? "MCSA with a device-built point Jacobi" : "MCSA";
        auto x = Teuchos::rcp(new TV(A->getRowMap()));
        auto b = Teuchos::rcp(new TV(A->getRowMap()));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<TV, TM>(A, x, b));
        MCLS::PointJacobiPreconditioner<TV, TM> pj;
        if (prec) {
            pj.setOperator(A);
            pj.buildPreconditioner();
            lp->setLeftPrec(pj.getLeftPreconditioner());
        }
        MCLS::SolverFactory<TV, TM> factory;
        auto sm = factory.create("Adjoint MCSA", pl);
        sm->setProblem(lp);
        for (double r : {-1.0, 2.0}) {
            fill(*b, r);
            fill(*x, 0.0);
            EXPECT(sm->solve() && sm->getNumIters() < 20);
            const auto xs = direct(rp, ci, v, std::vector<double>(size_t(n), r));
            double d = 0.0, s = 0.0;
            for (int i = 0; i < n; ++i) {
                const double xi = VT::view(*x)[i];
                EXPECT(r < 0 ? xi < 0.0 : xi > 0.0);
                d += (xi - xs[i]) * (xi - xs[i]);
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
