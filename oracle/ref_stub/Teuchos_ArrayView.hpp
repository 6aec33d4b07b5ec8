// Empty stand-in: the reference sampling header includes it but uses nothing.
#ifndef ORACLE_REF_STUB_TEUCHOS_ARRAYVIEW_HPP
#define ORACLE_REF_STUB_TEUCHOS_ARRAYVIEW_HPP
#endif
