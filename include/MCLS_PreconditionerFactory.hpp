// MCLS_PreconditionerFactory.hpp -- "Preconditioner Type" -> a device-built
// preconditioner, for LinearOpWithSolveFactory (MCLS_LinearOpWithSolve.hpp).
//
// Follows Thyra::MCLSPreconditionerFactory
// (thyra/src/Thyra_MCLSPreconditionerFactory_impl.hpp:58-330):
// "Preconditioner Type" (default "Point Jacobi") picks one sublist of
// "Preconditioner Types", whose entries configure that preconditioner.
// "Point Jacobi" and "Block Jacobi" ("Jacobi Block Size") are built on the
// device (MCLS_GpuPreconditioners.hpp); "Learned SPAI" is this library's
// own.  "ILUT", "ParaSails", "PSILUT" and "ML" wrap Ifpack, ParaSails and
// ML in the reference; those packages are not part of this library, and
// selecting one throws MCLS::Assertion when the preconditioner is created.
#ifndef MCLS_PRECONDITIONERFACTORY_HPP
#define MCLS_PRECONDITIONERFACTORY_HPP

#include <string>
#include <vector>

#include "MCLS_GpuPreconditioners.hpp"

namespace MCLS {

// What LinearOpWithSolveFactory needs of a preconditioner factory
// (Thyra::PreconditionerFactoryBase: createPrec, initializePrec,
// isCompatible).
template <class Matrix>
class PreconditionerFactoryBase : public virtual Teuchos::Describable {
  public:
    typedef Preconditioner<Matrix> Prec;
    virtual ~PreconditionerFactoryBase() = default;
    virtual bool isCompatible(const Matrix& A) const = 0;
    // A preconditioner of the configured type, not yet built.
    virtual Teuchos::RCP<Prec> createPrec() const = 0;
    // Builds `prec` for the operator A.
    virtual void initializePrec(const Teuchos::RCP<const Matrix>& A, Prec* prec) const = 0;
};

// A preconditioner built elsewhere (a Thyra preconditioner's operators, a
// user's own M^-1): its left and right matrices as given; either may be null.
template <class Matrix>
class GivenPreconditioner : public Preconditioner<Matrix> {
  public:
    GivenPreconditioner(const Teuchos::RCP<const Matrix>& left,
                        const Teuchos::RCP<const Matrix>& right)
        : d_left(left), d_right(right) {
        if (!Teuchos::nonnull(left) && !Teuchos::nonnull(right))
            throw Assertion("GivenPreconditioner: no left or right matrix");
    }
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        return Teuchos::parameterList();
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return Teuchos::parameterList();
    }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>&) override {}
    void setOperator(const Teuchos::RCP<const Matrix>& A) override { d_A = A; }
    const Matrix& getOperator() const override {
        if (!Teuchos::nonnull(d_A)) throw Assertion("GivenPreconditioner: no operator set");
        return *d_A;
    }
    void buildPreconditioner() override {}
    Teuchos::RCP<const Matrix> getLeftPreconditioner() const override { return d_left; }
    Teuchos::RCP<const Matrix> getRightPreconditioner() const override { return d_right; }
    std::string description() const override { return "MCLS::GivenPreconditioner"; }

  private:
    Teuchos::RCP<const Matrix> d_left, d_right, d_A;
};

template <class Vector, class Matrix>
class PreconditionerFactory : public PreconditionerFactoryBase<Matrix> {
  public:
    typedef Preconditioner<Matrix> Prec;
    typedef MatrixTraits<Vector, Matrix> MT;

    static constexpr const char* PrecType_name = "Preconditioner Type";
    static constexpr const char* PrecTypes_name = "Preconditioner Types";
    static constexpr const char* PrecType_default = "Point Jacobi";

    // The names the reference's factory accepts, then this library's own.
    static const std::vector<std::string>& precTypeNames() {
        static const std::vector<std::string> names = {
            "Point Jacobi", "Block Jacobi", "ILUT", "ParaSails", "PSILUT", "ML", "Learned SPAI"};
        return names;
    }

    PreconditionerFactory() : d_valid(makeValidParameters()) {}

    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const { return d_valid; }

    // Validates the list against getValidParameters() one sublist level deep
    // and fills in what is missing; an unknown "Preconditioner Type" throws
    // Teuchos::Exceptions::InvalidParameterValue.
    void setParameterList(const Teuchos::RCP<Teuchos::ParameterList>& params) {
        if (!Teuchos::nonnull(params))
            throw Assertion("PreconditionerFactory: null parameter list");
        params->validateParametersAndSetDefaults(*d_valid, 1);
        const std::string type = params->template get<std::string>(PrecType_name);
        bool known = false;
        for (const auto& n : precTypeNames()) known = known || n == type;
        if (!known)
            throw Teuchos::Exceptions::InvalidParameterValue(
                std::string("\"") + PrecType_name + "\" = \"" + type + "\" is not one of the " +
                "MCLS preconditioner types");
        d_plist = params;
        d_type = type;
    }
    Teuchos::RCP<Teuchos::ParameterList> getNonconstParameterList() { return d_plist; }
    Teuchos::RCP<const Teuchos::ParameterList> getParameterList() const { return d_plist; }
    Teuchos::RCP<Teuchos::ParameterList> unsetParameterList() {
        auto p = d_plist;
        d_plist = Teuchos::null;
        d_type = PrecType_default;
        return p;
    }
    const std::string& precType() const { return d_type; }

    bool isCompatible(const Matrix& A) const override { return MT::getGlobalNumRows(A) > 0; }

    Teuchos::RCP<Prec> createPrec() const override {
        auto sub = precParameters();
        if (d_type == "Point Jacobi")
            return Teuchos::rcp(new PointJacobiPreconditioner<Vector, Matrix>(sub));
        if (d_type == "Block Jacobi")
            return Teuchos::rcp(new BlockJacobiPreconditioner<Vector, Matrix>(sub));
        if (d_type == "Learned SPAI")
            return Teuchos::rcp(new LearnedSpaiPreconditioner<Vector, Matrix>(sub));
        const char* pkg = d_type == "ML" ? "ML" : (d_type == "ParaSails" ? "ParaSails" : "Ifpack");
        throw Assertion("Preconditioner Type \"" + d_type + "\" needs " + pkg +
                        ", which the GPU library does not provide");
    }
    void initializePrec(const Teuchos::RCP<const Matrix>& A, Prec* prec) const override {
        if (!Teuchos::nonnull(A) || prec == nullptr)
            throw Assertion("PreconditionerFactory::initializePrec: null operator or preconditioner");
        prec->setOperator(A);
        prec->buildPreconditioner();
    }

    std::string description() const override {
        return "MCLS::PreconditionerFactory{" + d_type + "}";
    }

  private:
    // The selected type's sublist of "Preconditioner Types" (kept alive with
    // the factory's list), or an empty list before setParameterList().
    Teuchos::RCP<Teuchos::ParameterList> precParameters() const {
        if (!Teuchos::nonnull(d_plist)) return Teuchos::parameterList();
        return Teuchos::sublist(Teuchos::sublist(d_plist, PrecTypes_name), d_type);
    }

    static Teuchos::RCP<const Teuchos::ParameterList> makeValidParameters() {
        auto pl = Teuchos::parameterList("MCLSPreconditionerFactory");
        pl->set<std::string>(PrecType_name, PrecType_default);
        Teuchos::ParameterList& types = pl->sublist(PrecTypes_name);
        types.sublist("Point Jacobi")
            .setParameters(*PointJacobiPreconditioner<Vector, Matrix>().getValidParameters());
        types.sublist("Block Jacobi")
            .setParameters(*BlockJacobiPreconditioner<Vector, Matrix>().getValidParameters());
        types.sublist("Learned SPAI")
            .setParameters(*LearnedSpaiPreconditioner<Vector, Matrix>().getValidParameters());
        // Ifpack's ILUT keys, kept so the reference's lists validate.
        types.sublist("ILUT").set<double>("fact: drop tolerance", 0.0);
        types.sublist("ILUT").set<double>("fact: ilut level-of-fill", 1.0);
        types.sublist("ParaSails");
        types.sublist("PSILUT");
        types.sublist("ML");
        return pl;
    }

    Teuchos::RCP<const Teuchos::ParameterList> d_valid;
    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    std::string d_type = PrecType_default;
};

}  // namespace MCLS

#endif  // MCLS_PRECONDITIONERFACTORY_HPP
