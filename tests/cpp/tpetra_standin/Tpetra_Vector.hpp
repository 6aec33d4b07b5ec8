#include "Tpetra_MultiVector.hpp"
