// Facade test: the MCLS manager API (SolverFactory, MCSASolverManager,
// MonteCarloSolverManager, LinearProblem, MultiSetLinearProblem,
// preconditioners, ParameterList keys) over libmclsgpu.
//
//   facade_test cpu   checks that need no device: valid parameter lists,
//                     factory names, ParameterList typing, LinearProblem's
//                     host helpers (tpetra/test/tstTpetraLinearProblem.cpp),
//                     and that a solve without a device throws MCLS::Assertion.
//   facade_test gpu   the solves, after the reference's manager tests
//                     (tpetra/test/tstTpetraMCSASolverManager.cpp:72-355,
//                     tpetra/test/tstTpetraMonteCarloSolverManager.cpp:73-197,
//                     tpetra/test/tstTpetraFixedPointSolverManager.cpp:72-345).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "MCLS_GpuPreconditioners.hpp"
#include "MCLS_SolverFactory.hpp"

typedef MCLS::HostVector Vec;
typedef MCLS::HostCrsMatrix Mat;
typedef MCLS::VectorTraits<Vec> VT;

static int g_failures = 0;
static std::string g_section = "start";
#define EXPECT(cond)                                                          \
    do {                                                                      \
        if (!(cond)) {                                                        \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);    \
            ++g_failures;                                                     \
        }                                                                     \
    } while (0)

// Tridiagonal (-0.14, 1, -0.14) with the explicit zeros of the reference test.
static Teuchos::RCP<Mat> tridiag(int n) {
    auto A = Teuchos::rcp(new Mat);
    A->n = n;
    A->rowptr.assign(1, 0);
    for (int i = 0; i < n; ++i) {
        int c0 = i == 0 ? 0 : (i == n - 1 ? n - 3 : i - 1);
        for (int c = c0; c < c0 + 3; ++c) {
            double v = c == i ? 1.0 : (std::abs(c - i) == 1 ? -0.14 : 0.0);
            A->colind.push_back(c);
            A->values.push_back(v);
        }
        A->rowptr.push_back(std::int64_t(A->colind.size()));
    }
    return A;
}

// Dense Gaussian elimination for the exact solution of a small system.
static Vec direct(const Mat& A, const Vec& b) {
    const int n = int(A.n);
    std::vector<double> M(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (auto p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p) M[size_t(i) * n + A.colind[p]] += A.values[p];
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

static Teuchos::RCP<Teuchos::ParameterList> mcsa_params() {
    auto pl = Teuchos::rcp(new Teuchos::ParameterList());
    pl->set<double>("Convergence Tolerance", 1.0e-8);
    pl->set<int>("Maximum Iterations", 20);
    pl->set<int>("MC Check Frequency", 50);
    pl->set<double>("Sample Ratio", 1.0);
    pl->set<std::string>("Transport Type", "Global");
    pl->set<bool>("Print Iterations", false);
    return pl;
}

static Teuchos::RCP<Mat> identity(int n) {
    auto I = Teuchos::rcp(new Mat);
    I->n = n;
    for (int i = 0; i < n; ++i) {
        I->colind.push_back(i);
        I->values.push_back(1.0);
        I->rowptr.push_back(i + 1);
    }
    return I;
}

static std::vector<double> dense(const Mat& A) {
    std::vector<double> D(size_t(A.n * A.n), 0.0);
    for (std::int64_t i = 0; i < A.n; ++i)
        for (auto p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p)
            D[size_t(i * A.n + A.colind[p])] += A.values[p];
    return D;
}

static std::vector<double> dense_mul(const std::vector<double>& X, const std::vector<double>& Y,
                                     int n, bool tx = false, bool ty = false) {
    std::vector<double> Z(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k)
                s += (tx ? X[size_t(k) * n + i] : X[size_t(i) * n + k]) *
                     (ty ? Y[size_t(j) * n + k] : Y[size_t(k) * n + j]);
            Z[size_t(i) * n + j] = s;
        }
    return Z;
}

// LinearProblem's host helpers, after tpetra/test/tstTpetraLinearProblem.cpp:
// Apply (:118-217), ResidualUpdate (:218-280), CompositeOperator (:281-330).
static void linear_problem_checks() {
    g_section = "LinearProblem apply";
    const int n = 10;
    {
        auto A = identity(n);
        auto X = Teuchos::rcp(new Vec(n, 2.0));
        auto B = Teuchos::rcp(new Vec(n, 5.0));
        MCLS::LinearProblem<Vec, Mat> lp(A, X, B);
        Vec Y(n, 0.0);
        lp.applyOp(*X, Y);
        for (double y : Y) EXPECT(y == 2.0);
        lp.updateSolution(X);  // the update aliases the LHS: X doubles
        lp.apply(*X, Y);
        for (double y : Y) EXPECT(y == 4.0);
        lp.setRightPrec(A);
        lp.applyRightPrec(*X, Y);
        for (double y : Y) EXPECT(y == 4.0);
        lp.apply(*X, Y);
        for (double y : Y) EXPECT(y == 4.0);
        lp.setLeftPrec(A);
        lp.applyLeftPrec(*X, Y);
        for (double y : Y) EXPECT(y == 4.0);
        lp.apply(*X, Y);
        for (double y : Y) EXPECT(y == 4.0);
        lp.updateSolution(X);
        auto composite = lp.getCompositeOperator();
        MCLS::MatrixTraits<Vec, Mat>::apply(*composite, *X, Y);
        for (double y : Y) EXPECT(y == 8.0);
    }
    g_section = "LinearProblem residual update";
    {
        auto A = identity(n);
        auto X = Teuchos::rcp(new Vec(n, 2.0));
        auto B = Teuchos::rcp(new Vec(n, 5.0));
        MCLS::LinearProblem<Vec, Mat> lp(A, X, B);
        lp.updateResidual();
        for (double r : *lp.getResidual()) EXPECT(r == 3.0);
        for (double r : *lp.getPrecResidual()) EXPECT(r == 0.0);
        lp.setLeftPrec(A);
        lp.updateResidual();
        for (double r : *lp.getResidual()) EXPECT(r == 3.0);
        lp.updatePrecResidual();
        for (double r : *lp.getPrecResidual()) EXPECT(r == 3.0);
    }
    g_section = "LinearProblem composite operator";
    {
        // A: 1 on the diagonal and 2 right of it, last row empty; PL = A^T:
        // interior rows of PL A are (2, 5, 2).
        auto A = Teuchos::rcp(new Mat);
        A->n = n;
        for (int i = 0; i < n - 1; ++i) {
            A->colind.push_back(i);
            A->values.push_back(1.0);
            A->colind.push_back(i + 1);
            A->values.push_back(2.0);
            A->rowptr.push_back(std::int64_t(A->colind.size()));
        }
        A->rowptr.push_back(std::int64_t(A->colind.size()));
        auto X = Teuchos::rcp(new Vec(n, 2.0));
        MCLS::LinearProblem<Vec, Mat> lp0(A, X, X);
        EXPECT(lp0.getCompositeOperator() == A);  // no preconditioner: A itself
        MCLS::LinearProblem<Vec, Mat> tp(A, X, X);
        auto C = tp.getTransposeCompositeOperator();
        MCLS::LinearProblem<Vec, Mat> lp(A, X, X);
        lp.setLeftPrec(C);
        auto D = lp.getCompositeOperator();
        for (int i = 1; i < n - 1; ++i) {
            EXPECT(D->rowptr[i + 1] - D->rowptr[i] == 3);
            const auto p = D->rowptr[i];
            EXPECT(D->colind[p] == i - 1 && D->colind[p + 1] == i && D->colind[p + 2] == i + 1);
            EXPECT(D->values[p] == 2.0 && D->values[p + 1] == 5.0 && D->values[p + 2] == 2.0);
        }
        // Both preconditioners, and the transposed composite, against dense
        // products of a nonsymmetric case; the threshold drops the small
        // products of each row.
        auto T = tridiag(n);
        auto P = Teuchos::rcp(new Mat(*T));
        for (auto& v : P->values) v = v == 1.0 ? 0.5 : v * 3.0;
        MCLS::LinearProblem<Vec, Mat> both(A, X, X);
        both.setLeftPrec(T);
        both.setRightPrec(P);
        const auto dA = dense(*A), dT = dense(*T), dP = dense(*P);
        const auto ref = dense_mul(dT, dense_mul(dA, dP, n), n);
        const auto got = dense(*both.getCompositeOperator());
        const auto gotT = dense(*both.getTransposeCompositeOperator());
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                EXPECT(std::fabs(got[size_t(i) * n + j] - ref[size_t(i) * n + j]) < 1e-14);
                EXPECT(std::fabs(gotT[size_t(j) * n + i] - ref[size_t(i) * n + j]) < 1e-14);
            }
        // Each product is filtered (|c| <= 0.3 * signed row max and zeros
        // dropped) before the next one, as the reference's multiply does.
        auto filt = [n](std::vector<double> M) {
            for (int i = 0; i < n; ++i) {
                double rmax = 0.0;
                bool first = true;
                for (int j = 0; j < n; ++j)
                    if (M[size_t(i) * n + j] != 0.0) {
                        rmax = first ? M[size_t(i) * n + j] : std::max(rmax, M[size_t(i) * n + j]);
                        first = false;
                    }
                for (int j = 0; j < n; ++j)
                    if (std::fabs(M[size_t(i) * n + j]) <= 0.3 * rmax) M[size_t(i) * n + j] = 0.0;
            }
            return M;
        };
        const auto reff = filt(dense_mul(dT, filt(dense_mul(dA, dP, n)), n));
        auto F = both.getCompositeOperator(0.3);
        const auto gotf = dense(*F);
        int kept = 0;
        for (int i = 0; i < n * n; ++i) {
            EXPECT(std::fabs(gotf[size_t(i)] - reff[size_t(i)]) < 1e-14);
            kept += reff[size_t(i)] != 0.0;
        }
        int unfiltered = 0;
        for (double r : ref) unfiltered += r != 0.0;
        EXPECT(std::int64_t(F->values.size()) == kept && kept < unfiltered);
    }
}

static void cpu_checks() {
    linear_problem_checks();
    MCLS::SolverFactory<Vec, Mat> factory;
    auto pl = mcsa_params();
    for (const char* name : {"Adjoint MC", "Forward MC", "Adjoint MCSA", "Forward MCSA"}) {
        auto s = factory.create(name, pl);
        EXPECT(Teuchos::nonnull(s));
        auto v = s->getValidParameters();
        EXPECT(v->isParameter("Sample Ratio") && v->isParameter("History Length"));
        EXPECT(v->isParameter("Neumann Relaxation") && v->isParameter("MC Check Frequency"));
        EXPECT(s->getCurrentParameters() == pl);
    }
    auto mcsa = factory.create("Adjoint MCSA", pl);
    auto v = mcsa->getValidParameters();
    EXPECT(v->get<double>("Convergence Tolerance") == 1.0);
    EXPECT(v->get<int>("Maximum Iterations") == 1000);
    EXPECT(v->get<std::string>("Fixed Point Type") == "Richardson");
    auto fp = factory.create("Fixed Point", pl);
    EXPECT(Teuchos::nonnull(fp));
    EXPECT(fp->getValidParameters()->get<std::string>("Fixed Point Type") == "Richardson");
    EXPECT(fp->getValidParameters()->get<double>("Richardson Relaxation") == 1.0);
    for (const char* name : {"Adjoint Anderson", "Forward Anderson"}) {
        auto a = factory.create(name, pl);
        EXPECT(Teuchos::nonnull(a));
        auto va = a->getValidParameters();
        EXPECT(va->get<double>("Convergence Tolerance") == 1.0e-8);
        EXPECT(va->sublist("Anderson Parameters").get<int>("Storage Depth") == 2);
        EXPECT(pl->get<std::string>("Nonlinear Solver") == "Anderson Accelerated Fixed-Point");
    }
    {
        auto bad = mcsa_params();
        bad->sublist("Anderson Parameters").set<int>("Storage Depth", 40);
        bool threw = false;
        try {
            factory.create("Adjoint Anderson", bad);
        } catch (const MCLS::Assertion&) {
            threw = true;
        }
        EXPECT(threw);
    }
    for (const char* name : {"Bogus"}) {
        bool threw = false;
        try {
            factory.create(name, pl);
        } catch (const MCLS::Assertion&) {
            threw = true;
        }
        EXPECT(threw);
    }
    for (const char* type : {"Richardson", "Steepest Descent", "MINRES", "RNSD"}) {
        auto ok = mcsa_params();
        ok->set<std::string>("Fixed Point Type", type);
        MCLS::MCSASolverManager<Vec, Mat> m(ok);
        MCLS::FixedPointSolverManager<Vec, Mat> f(ok);
    }
    bool threw = false;
    try {
        auto bad = mcsa_params();
        bad->set<std::string>("Fixed Point Type", "Jacobi");
        MCLS::MCSASolverManager<Vec, Mat> m(bad);
    } catch (const MCLS::Assertion& e) {
        threw = std::string(e.what()).find("Iteration type not supported!") != std::string::npos;
    }
    EXPECT(threw);
    // Teuchos-strict typing.
    threw = false;
    try {
        pl->get<int>("Sample Ratio");
    } catch (const Teuchos::Exceptions::InvalidParameterType&) {
        threw = true;
    }
    EXPECT(threw);
    EXPECT(pl->get<int>("Smoother Steps", 1) == 1 && pl->isParameter("Smoother Steps"));

    // A solve with no device reports it through MCLS::Assertion.
    auto A = tridiag(10);
    auto x = Teuchos::rcp(new Vec(10, 0.0));
    auto b = Teuchos::rcp(new Vec(10, -1.0));
    auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
    mcsa->setProblem(lp);
    std::string msg;
    try {
        mcsa->solve();
    } catch (const MCLS::Assertion& e) {
        msg = e.what();
    }
    EXPECT(msg.find("no usable CUDA device") != std::string::npos);
}

static void gpu_checks() {
    const int n = 10;
    auto A = tridiag(n);
    auto comm = Teuchos::DefaultComm<int>::getComm();
    for (int forward = 0; forward < 2; ++forward) {
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, -1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
        auto ms = Teuchos::rcp(new MCLS::MultiSetLinearProblem<Vec, Mat>(comm, 1, 0, lp));
        auto pl = mcsa_params();
        if (forward) pl->set<double>("Sample Ratio", 10.0);
        Teuchos::RCP<MCLS::SolverManager<Vec, Mat>> sm;
        if (forward)
            sm = Teuchos::rcp(new MCLS::MCSASolverManager<Vec, Mat, MCLS::ForwardTag>(ms, pl));
        else
            sm = Teuchos::rcp(new MCLS::MCSASolverManager<Vec, Mat, MCLS::AdjointTag>(ms, pl));
        const double rhs[4] = {-1.0, 2.0, -2.0, 1.0};
        for (double r : rhs) {  // four successive solves on one manager
            g_section = std::string(forward ? "forward" : "adjoint") + " MCSA, b = " +
                        std::to_string(r);
            std::fill(b->begin(), b->end(), r);
            std::fill(x->begin(), x->end(), 0.0);
            lp->setLHS(x);
            bool conv = sm->solve();
            EXPECT(conv && sm->getConvergedStatus());
            EXPECT(sm->getNumIters() < 20);
            EXPECT(sm->achievedTol() > 0.0 && sm->achievedTol() <= 1e-8);
            for (double xi : *x) EXPECT(r < 0 ? xi < 0.0 : xi > 0.0);
            EXPECT(rel_err(*x, direct(*A, *b)) < 1e-7);
        }
    }

    // Left point-Jacobi built on the device and handed to the problem.
    {
        g_section = "point Jacobi";
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, 2.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
        MCLS::PointJacobiPreconditioner<Vec, Mat> prec;
        prec.setOperator(A);
        prec.buildPreconditioner();
        auto PL = prec.getLeftPreconditioner();
        EXPECT(Teuchos::nonnull(PL) && PL->n == n && PL->values.size() == size_t(n));
        EXPECT(std::fabs(PL->values[3] - 1.0) < 1e-15);
        lp->setLeftPrec(PL);
        MCLS::SolverFactory<Vec, Mat> factory;
        auto pl = mcsa_params();
        auto sm = factory.create("Adjoint MCSA", pl);
        sm->setProblem(lp);
        EXPECT(sm->solve());
        EXPECT(rel_err(*x, direct(*A, *b)) < 1e-7);
    }

    // Block Jacobi (blocks of 2) on a matrix with a non-unit diagonal.
    {
        g_section = "block Jacobi";
        auto B = tridiag(n);
        for (int i = 0; i < n; ++i)
            for (auto p = B->rowptr[i]; p < B->rowptr[i + 1]; ++p)
                if (B->colind[p] == i) B->values[p] = 2.0 + 0.1 * i;
        auto params = Teuchos::parameterList();
        params->set<int>("Jacobi Block Size", 2);
        MCLS::BlockJacobiPreconditioner<Vec, Mat> prec(params);
        prec.setOperator(B);
        prec.buildPreconditioner();
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, 1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(B, x, b));
        lp->setLeftPrec(prec.getLeftPreconditioner());
        // Forward: with blocks of 2, H = I - PL A has columns that vanish
        // (a column of A inside one diagonal block), which the adjoint domain
        // rejects as the reference does (MCLS_CHECK on empty rows of H^T).
        auto pl = mcsa_params();
        pl->set<double>("Sample Ratio", 10.0);
        MCLS::MCSASolverManager<Vec, Mat, MCLS::ForwardTag> sm(pl);
        sm.setProblem(lp);
        EXPECT(sm.solve());
        EXPECT(rel_err(*x, direct(*B, *b)) < 1e-7);
    }

    // The reference's block inversion known answer
    // (test/tstBlockInversion.cpp:46-105) through a block of size 4.
    {
        g_section = "block inversion";
        const double B[16] = {3.2,  -1.43, 2.98, 0.32,  -4.12, -7.53, 1.44, -3.72,
                              4.24, -6.42, 1.82, 2.67, -0.23, 5.8,   1.13, -3.73};
        const double inv[16] = {-0.461356423424245, -0.060920073472551, 0.547244760641934,
                                0.412904055961420,  0.154767451798665,  -0.056225122550555,
                                -0.174451348828054, -0.055523340725809, 0.848746201780808,
                                0.045927762119214,  -0.618485718805259, -0.415712965073367,
                                0.526232280383953,  -0.069757566407458, -0.492378815120724,
                                -0.505833501236923};
        auto M4 = Teuchos::rcp(new Mat);
        M4->n = 4;
        for (int i = 0; i < 4; ++i) {
            for (int j = 0; j < 4; ++j) {
                M4->colind.push_back(j);
                M4->values.push_back(B[4 * i + j]);
            }
            M4->rowptr.push_back(4 * (i + 1));
        }
        auto params = Teuchos::parameterList();
        params->set<int>("Jacobi Block Size", 4);
        MCLS::BlockJacobiPreconditioner<Vec, Mat> prec(params);
        prec.setOperator(M4);
        prec.buildPreconditioner();
        auto PL = prec.getLeftPreconditioner();
        EXPECT(PL->n == 4 && PL->values.size() == 16);
        double got[16] = {0};
        for (int i = 0; i < 4; ++i)
            for (auto p = PL->rowptr[i]; p < PL->rowptr[i + 1]; ++p)
                got[4 * i + PL->colind[p]] = PL->values[p];
        for (int k = 0; k < 16; ++k) EXPECT(std::fabs(got[k] - inv[k]) <= 1e-13 * std::fabs(inv[k]));
    }

    // Learned SPAI with a network whose output layer is zero: M is point
    // Jacobi, the rho gate keeps the plain preconditioner, the solve converges.
    {
        g_section = "learned SPAI";
        const int m = 8, N = m * m;
        auto P2 = Teuchos::rcp(new Mat);
        P2->n = N;
        P2->rowptr.assign(1, 0);
        for (int i = 0; i < N; ++i) {
            const int x = i % m, y = i / m;
            const int nb[5] = {y > 0 ? i - m : -1, x > 0 ? i - 1 : -1, i, x < m - 1 ? i + 1 : -1,
                               y < m - 1 ? i + m : -1};
            for (int c : nb)
                if (c >= 0) {
                    P2->colind.push_back(c);
                    P2->values.push_back(c == i ? 4.0 : -1.0);
                }
            P2->rowptr.push_back(std::int64_t(P2->colind.size()));
        }
        std::vector<float> w(size_t(mclsgpu_spai_num_params()), 0.0f);
        auto sp = Teuchos::parameterList();
        sp->set<std::vector<float>>("SPAI Weights", w);
        MCLS::LearnedSpaiPreconditioner<Vec, Mat> prec(sp);
        prec.setOperator(P2);
        prec.buildPreconditioner();
        auto PL = prec.getLeftPreconditioner();
        // Kept on A's pattern (rho below the gate) or replaced by point
        // Jacobi: either way 1/4 on the diagonal and zero elsewhere.
        EXPECT(Teuchos::nonnull(PL) && PL->n == N);
        for (int i = 0; i < N; ++i)
            for (auto p = PL->rowptr[i]; p < PL->rowptr[i + 1]; ++p)
                EXPECT(std::fabs(PL->values[p] - (PL->colind[p] == i ? 0.25 : 0.0)) < 1e-15);
        auto x = Teuchos::rcp(new Vec(N, 0.0));
        auto b = Teuchos::rcp(new Vec(N, 1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(P2, x, b));
        lp->setLeftPrec(PL);
        auto pl = mcsa_params();
        pl->set<int>("Maximum Iterations", 2000);
        MCLS::MCSASolverManager<Vec, Mat> sm(pl);
        sm.setProblem(lp);
        EXPECT(sm.solve());
        EXPECT(rel_err(*x, direct(*P2, *b)) < 1e-7);
    }

    // Fixed point, Richardson: exactly 15 iterations, the solution's sign
    // follows the source, also with PL = PR = I
    // (tpetra/test/tstTpetraFixedPointSolverManager.cpp:72-345).
    {
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
        auto I = Teuchos::rcp(new Mat);
        I->n = n;
        I->rowptr.assign(1, 0);
        for (int i = 0; i < n; ++i) {
            I->colind.push_back(i);
            I->values.push_back(1.0);
            I->rowptr.push_back(i + 1);
        }
        for (int prec = 0; prec < 2; ++prec) {
            auto x = Teuchos::rcp(new Vec(n, 0.0));
            auto b = Teuchos::rcp(new Vec(n, -1.0));
            auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(F, x, b));
            if (prec) {
                lp->setLeftPrec(I);
                lp->setRightPrec(I);
            }
            auto pl = Teuchos::parameterList();
            pl->set<int>("Iteration Print Frequency", 1);
            pl->set<double>("Convergence Tolerance", 1.0e-8);
            pl->set<int>("Maximum Iterations", 100);
            pl->set<double>("Richardson Relaxation", 1.0);
            pl->set<bool>("Print Iterations", false);
            MCLS::FixedPointSolverManager<Vec, Mat> sm(lp, pl);
            for (double r : {-1.0, 2.0, 2.0, -2.0}) {
                g_section = std::string("fixed point, b = ") + std::to_string(r);
                std::fill(b->begin(), b->end(), r);
                std::fill(x->begin(), x->end(), 0.0);
                lp->setLHS(x);
                sm.setProblem(lp);
                EXPECT(sm.solve() && sm.getConvergedStatus());
                EXPECT(sm.getNumIters() == 15);
                EXPECT(sm.achievedTol() > 0.0);
                for (double xi : *x) EXPECT(r < 0 ? xi < 0.0 : xi > 0.0);
            }
        }
        // MCSA with a MINRES smoother through the factory.
        g_section = "MCSA with MINRES smoother";
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, -1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
        auto pl = mcsa_params();
        pl->set<std::string>("Fixed Point Type", "MINRES");
        MCLS::SolverFactory<Vec, Mat> factory;
        auto sm = factory.create("Adjoint MCSA", pl);
        sm->setProblem(lp);
        EXPECT(sm->solve() && sm->getNumIters() < 20);
        EXPECT(rel_err(*x, direct(*A, *b)) < 1e-7);
    }

    // Anderson-accelerated MCSA: the reference's MCSA checks (signs, the
    // direct solution) through the "Adjoint/Forward Anderson" managers, with
    // the NOX sublist.
    for (const char* name : {"Adjoint Anderson", "Forward Anderson"}) {
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, -1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
        auto ms = Teuchos::rcp(new MCLS::MultiSetLinearProblem<Vec, Mat>(comm, 1, 0, lp));
        auto pl = mcsa_params();
        pl->set<int>("Maximum Iterations", 100);
        pl->set<double>("Sample Ratio", 10.0);
        pl->sublist("Anderson Parameters").set<int>("Storage Depth", 3);
        MCLS::SolverFactory<Vec, Mat> factory;
        auto sm = factory.create(name, pl);
        for (double r : {-1.0, 2.0}) {
            g_section = std::string(name) + ", b = " + std::to_string(r);
            std::fill(b->begin(), b->end(), r);
            std::fill(x->begin(), x->end(), 0.0);
            sm->setProblem(lp);
            EXPECT(sm->solve() && sm->getConvergedStatus());
            EXPECT(sm->getNumIters() > 0 && sm->getNumIters() < 100);
            EXPECT(sm->achievedTol() < 1e-8);
            for (double xi : *x) EXPECT(r < 0 ? xi < 0.0 : xi > 0.0);
            EXPECT(rel_err(*x, direct(*A, *b)) < 1e-7);
        }
    }

    // Direct Monte Carlo: signs follow the source, sample ratio 10
    // (tpetra/test/tstTpetraMonteCarloSolverManager.cpp:73-197).
    for (const char* name : {"Adjoint MC", "Forward MC"}) {
        g_section = name;
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, -1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
        auto pl = Teuchos::parameterList();
        pl->set<double>("Sample Ratio", 10.0);
        MCLS::SolverFactory<Vec, Mat> factory;
        auto sm = factory.create(name, pl);
        sm->setProblem(lp);
        EXPECT(sm->solve() && sm->getConvergedStatus() && sm->getNumIters() == 0);
        for (double xi : *x) EXPECT(xi < 0.0);
        // |b - A x|_inf / |b|_inf: the stochastic error of one direct solve
        // with 100 histories (the reference tests check signs only).
        EXPECT(std::isfinite(sm->achievedTol()) && sm->achievedTol() > 0.0);
        std::fill(b->begin(), b->end(), 2.0);
        sm->solve();
        for (double xi : *x) EXPECT(xi > 0.0);
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
