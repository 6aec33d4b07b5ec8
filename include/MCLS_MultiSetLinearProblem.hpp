// MCLS_MultiSetLinearProblem.hpp -- the set decomposition handle the MCSA
// manager accepts (src/MCLS_MultiSetLinearProblem_impl.hpp:56-120).
//
// On the GPU path one process (or host thread) drives one set on one device.
// With several sets the manager sums their Monte Carlo corrections every
// iteration through the set reducer this handle carries
// (MultiSetLinearProblem::blockConstantVectorSum,
// src/MCLS_MultiSetLinearProblem_impl.hpp:102-120): the library's NCCL
// communicator (mclsgpu_comm_set_params; the loop then stays on the device)
// or any caller-supplied sum over the sets (an MPI all-reduce on host copies,
// say; the loop then runs from the host).
#ifndef MCLS_MULTISETLINEARPROBLEM_HPP
#define MCLS_MULTISETLINEARPROBLEM_HPP

#include "MCLS_LinearProblem.hpp"
#include "mclsgpu.h"

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

    // The reducer that sums the sets' corrections (required when
    // getNumSets() > 1).  See mclsgpu_set_params.
    void setSetReducer(const mclsgpu_set_params& sets) {
        if (sets.num_sets != d_num_sets || !sets.reduce)
            throw Assertion("MultiSetLinearProblem: reducer of another set count");
        d_sets = sets;
        d_has_sets = true;
    }
    bool hasSetReducer() const { return d_has_sets; }
    const mclsgpu_set_params& setReducer() const { return d_sets; }

    Teuchos::RCP<LinearProblemType> getProblem() const { return d_problem; }
    Teuchos::RCP<const Teuchos::Comm<int>> getGlobalComm() const { return d_comm; }
    int getNumSets() const { return d_num_sets; }
    int getSetID() const { return d_set_id; }

  private:
    Teuchos::RCP<const Teuchos::Comm<int>> d_comm;
    int d_num_sets;
    int d_set_id;
    Teuchos::RCP<LinearProblemType> d_problem;
    mclsgpu_set_params d_sets{};
    bool d_has_sets = false;
};

}  // namespace MCLS

#endif  // MCLS_MULTISETLINEARPROBLEM_HPP
