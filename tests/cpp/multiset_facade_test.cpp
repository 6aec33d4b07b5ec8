// Multi-set MCSA through the C++ manager API: two sets of one problem, each
// driven by its own host thread and MCSASolverManager on one GPU, with a
// MultiSetLinearProblem of two sets whose set reducer sums the two sets'
// Monte Carlo corrections on the host (the form an MPI all-reduce of host
// copies takes; no kernel waits on the other set).  "Number of Sets" = 2.
// Checks: both sets converge in the same number of iterations to the same
// iterate, equal to the direct solution; a problem of two sets without a
// reducer, or a "Number of Sets" that disagrees, throws MCLS::Assertion.
#include <cuda_runtime.h>

#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "MCLS_SolverFactory.hpp"

typedef MCLS::HostVector Vec;
typedef MCLS::HostCrsMatrix Mat;

static int g_failures = 0;
#define EXPECT(cond)                                                       \
    do {                                                                   \
        if (!(cond)) {                                                     \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            ++g_failures;                                                  \
        }                                                                  \
    } while (0)

// 2D Poisson 5-point on an m x m grid with its rows scaled to a unit
// diagonal (1 on the diagonal, -1/4 beside it), so that the iteration matrix
// I - A of the unpreconditioned problem has spectral radius cos(pi/(m+1)) < 1.
static Teuchos::RCP<Mat> poisson(int m) {
    auto A = Teuchos::rcp(new Mat);
    A->n = m * m;
    A->rowptr.assign(1, 0);
    for (int y = 0; y < m; ++y)
        for (int x = 0; x < m; ++x) {
            const int i = y * m + x;
            auto put = [&](int c, double v) {
                A->colind.push_back(c);
                A->values.push_back(v);
            };
            if (y > 0) put(i - m, -0.25);
            if (x > 0) put(i - 1, -0.25);
            put(i, 1.0);
            if (x < m - 1) put(i + 1, -0.25);
            if (y < m - 1) put(i + m, -0.25);
            A->rowptr.push_back(std::int64_t(A->colind.size()));
        }
    return A;
}

// In-process sum over two sets: each set copies its correction to the host,
// both wait for each other, each adds the two copies in set order and copies
// the sum back.
struct TwoSetSum {
    std::mutex m;
    std::condition_variable cv;
    std::vector<double> slot[2];
    int arrived = 0, generation = 0, left = 0;

    void wait_all() {
        std::unique_lock<std::mutex> lk(m);
        const int g = generation;
        if (++arrived == 2) {
            arrived = 0;
            ++generation;
            cv.notify_all();
        } else {
            cv.wait(lk, [&] { return generation != g; });
        }
    }
};

struct SetUser {
    TwoSetSum* sum;
    int set;
};

static int reduce_two(void* user, double* data, int64_t n, void* stream) {
    SetUser* u = static_cast<SetUser*>(user);
    std::vector<double>& mine = u->sum->slot[u->set];
    mine.resize(size_t(n));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Both copies on the set's stream, each completed before the host goes on
    // (the stream does not synchronise with the legacy default stream).
    if (cudaMemcpyAsync(mine.data(), data, size_t(n) * 8, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return 2;
    u->sum->wait_all();
    std::vector<double> total(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) total[i] = u->sum->slot[0][i] + u->sum->slot[1][i];
    u->sum->wait_all();  // both have read the slots before the next iteration
    if (cudaMemcpyAsync(data, total.data(), size_t(n) * 8, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return 2;
    return 0;
}

int main() {
    const int m = 12, n = m * m;
    auto A = poisson(m);
    auto comm = Teuchos::DefaultComm<int>::getComm();
    TwoSetSum sum;
    SetUser users[2] = {{&sum, 0}, {&sum, 1}};
    Vec xs[2];
    int iters[2] = {0, 0};
    bool conv[2] = {false, false};
    std::string errors[2];
    auto run = [&](int set) {
        try {
            auto x = Teuchos::rcp(new Vec(n, 0.0));
            auto b = Teuchos::rcp(new Vec(n, 1.0));
            auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
            auto ms = Teuchos::rcp(new MCLS::MultiSetLinearProblem<Vec, Mat>(comm, 2, set, lp));
            mclsgpu_set_params sp{};
            sp.size = sizeof(sp);
            sp.num_sets = 2;
            sp.reduce = &reduce_two;
            sp.user = &users[set];
            ms->setSetReducer(sp);
            auto pl = Teuchos::parameterList();
            pl->set<double>("Convergence Tolerance", 1e-8);
            pl->set<int>("Maximum Iterations", 2000);
            pl->set<double>("Sample Ratio", 4.0);
            pl->set<int>("Number of Sets", 2);
            pl->set<double>("Random Seed", 1000.0 + 17.0 * set);
            MCLS::MCSASolverManager<Vec, Mat> sm(ms, pl);
            conv[set] = sm.solve();
            iters[set] = sm.getNumIters();
            xs[set] = *x;
        } catch (const std::exception& e) {
            errors[set] = e.what();
        }
    };
    std::thread t1(run, 1);
    run(0);
    t1.join();
    for (int s = 0; s < 2; ++s)
        if (!errors[s].empty()) std::printf("set %d: %s\n", s, errors[s].c_str());
    EXPECT(errors[0].empty() && errors[1].empty());
    EXPECT(conv[0] && conv[1]);
    EXPECT(iters[0] == iters[1] && iters[0] > 0);
    EXPECT(xs[0] == xs[1]);
    // Against the exact solution of A x = 1 (a tight CG on the host).
    {
        Vec x(n, 0.0), r(n, 1.0), p(n, 1.0), q(n);
        double rr = n;
        for (int it = 0; it < 1000 && rr > 1e-28; ++it) {
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (auto k = A->rowptr[i]; k < A->rowptr[i + 1]; ++k) s += A->values[k] * p[A->colind[k]];
                q[i] = s;
            }
            double pq = 0;
            for (int i = 0; i < n; ++i) pq += p[i] * q[i];
            const double a = rr / pq;
            double rr2 = 0;
            for (int i = 0; i < n; ++i) {
                x[i] += a * p[i];
                r[i] -= a * q[i];
                rr2 += r[i] * r[i];
            }
            for (int i = 0; i < n; ++i) p[i] = r[i] + rr2 / rr * p[i];
            rr = rr2;
        }
        double d = 0, nn = 0;
        for (int i = 0; i < n; ++i) {
            d += (xs[0][i] - x[i]) * (xs[0][i] - x[i]);
            nn += x[i] * x[i];
        }
        EXPECT(std::sqrt(d / nn) < 1e-6);
    }
    // The Anderson-accelerated manager on the same two sets.
    {
        Vec xa[2];
        bool aconv[2] = {false, false};
        int aiters[2] = {0, 0};
        auto run_aa = [&](int set) {
            try {
                auto x = Teuchos::rcp(new Vec(n, 0.0));
                auto b = Teuchos::rcp(new Vec(n, 1.0));
                auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
                auto ms = Teuchos::rcp(new MCLS::MultiSetLinearProblem<Vec, Mat>(comm, 2, set, lp));
                mclsgpu_set_params sp{};
                sp.size = sizeof(sp);
                sp.num_sets = 2;
                sp.reduce = &reduce_two;
                sp.user = &users[set];
                ms->setSetReducer(sp);
                auto pl = Teuchos::parameterList();
                pl->set<double>("Convergence Tolerance", 1e-8);
                pl->set<int>("Maximum Iterations", 2000);
                pl->set<double>("Sample Ratio", 4.0);
                pl->set<int>("Number of Sets", 2);
                pl->set<double>("Random Seed", 5000.0 + 31.0 * set);
                pl->sublist("Anderson Parameters").set<int>("Storage Depth", 3);
                MCLS::AndersonSolverManager<Vec, Mat> sm(ms, pl);
                aconv[set] = sm.solve();
                aiters[set] = sm.getNumIters();
                xa[set] = *x;
            } catch (const std::exception& e) {
                errors[set] = e.what();
            }
        };
        std::thread t2(run_aa, 1);
        run_aa(0);
        t2.join();
        for (int s2 = 0; s2 < 2; ++s2)
            if (!errors[s2].empty()) std::printf("anderson set %d: %s\n", s2, errors[s2].c_str());
        EXPECT(aconv[0] && aconv[1]);
        EXPECT(aiters[0] == aiters[1] && aiters[0] > 0);
        EXPECT(xa[0] == xa[1]);
    }
    // Two sets without a reducer, or a "Number of Sets" that disagrees.
    {
        auto x = Teuchos::rcp(new Vec(n, 0.0));
        auto b = Teuchos::rcp(new Vec(n, 1.0));
        auto lp = Teuchos::rcp(new MCLS::LinearProblem<Vec, Mat>(A, x, b));
        auto ms2 = Teuchos::rcp(new MCLS::MultiSetLinearProblem<Vec, Mat>(comm, 2, 0, lp));
        auto pl = Teuchos::parameterList();
        bool threw = false;
        try {
            MCLS::MCSASolverManager<Vec, Mat> sm(ms2, pl);
        } catch (const MCLS::Assertion&) {
            threw = true;
        }
        EXPECT(threw);
        auto ms1 = Teuchos::rcp(new MCLS::MultiSetLinearProblem<Vec, Mat>(comm, 1, 0, lp));
        pl->set<int>("Number of Sets", 2);
        threw = false;
        try {
            MCLS::MCSASolverManager<Vec, Mat> sm(ms1, pl);
            sm.solve();
        } catch (const MCLS::Assertion&) {
            threw = true;
        }
        EXPECT(threw);
    }
    std::printf("multiset: %d failure(s)\n", g_failures);
    return g_failures ? 1 : 0;
}
