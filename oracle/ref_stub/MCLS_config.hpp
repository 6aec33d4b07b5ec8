// Configuration of the reference build used by oracle/_ref: design-by-contract
// and timers off (the reference's production setting).
#define HAVE_MCLS_DBC 0
#define HAVE_MCLS_TIMERS 0
#define HAVE_MCLS_PARASAILS 0
#define HAVE_MCLS_EPETRA 0
#define HAVE_MCLS_TEMERE 0
