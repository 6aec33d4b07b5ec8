// MCLS_MultiSetLinearProblem.hpp -- the set decomposition handle the MCSA
// manager accepts (src/MCLS_MultiSetLinearProblem_impl.hpp:56-120).
//
// On the GPU path one process drives one device and one set.  Several sets
// (one per GPU) sum their Monte Carlo corrections with an all-reduce in the
// Python multi-set driver; this C++ handle carries the set layout and the
// set's LinearProblem.
#ifndef MCLS_MULTISETLINEARPROBLEM_HPP
#define MCLS_MULTISETLINEARPROBLEM_HPP

#include "MCLS_LinearProblem.hpp"

namespace MCLS {

template <class Vector, class Matrix>
class MultiSetLinearProblem {
  public:
    typedef LinearProblem<Vector, Matrix> LinearProblemType;

    MultiSetLinearProblem(const Teuchos::RCP<const Teuchos::Comm<int>>& global_comm, int num_sets,
                          int set_id, const Teuchos::RCP<LinearProblemType>& problem)
        : d_comm(global_comm), d_num_sets(num_sets), d_set_id(set_id), d_problem(problem) {
        if (num_sets < 1 || set_id < 0 || set_id >= num_sets)
            throw Assertion("MultiSetLinearProblem: bad set layout");
        if (!Teuchos::nonnull(problem)) throw Assertion("MultiSetLinearProblem: null problem");
    }
    MultiSetLinearProblem(const Teuchos::RCP<const Teuchos::Comm<int>>& global_comm, int num_sets,
                          int set_id, const Teuchos::RCP<const Matrix>& A,
                          const Teuchos::RCP<Vector>& x, const Teuchos::RCP<const Vector>& b)
        : MultiSetLinearProblem(global_comm, num_sets, set_id,
                                Teuchos::rcp(new LinearProblemType(A, x, b))) {}

    Teuchos::RCP<LinearProblemType> getProblem() const { return d_problem; }
    Teuchos::RCP<const Teuchos::Comm<int>> getGlobalComm() const { return d_comm; }
    int getNumSets() const { return d_num_sets; }
    int getSetID() const { return d_set_id; }

  private:
    Teuchos::RCP<const Teuchos::Comm<int>> d_comm;
    int d_num_sets;
    int d_set_id;
    Teuchos::RCP<LinearProblemType> d_problem;
};

}  // namespace MCLS

#endif  // MCLS_MULTISETLINEARPROBLEM_HPP
