// oracle/shim/mkl_lapack.h — TEST INFRASTRUCTURE ONLY: everything lives in mkl.h.
#include "mkl.h"
