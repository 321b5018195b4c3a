// ref_app.cpp -- builds one of the reference's iterative-solver applications,
// UNMODIFIED, as a CPU program.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file with
// -DSMAX_APP_SOURCE="<path of examples/applications/{jacobi,gauss_seidel}/*.cpp>"
// into oracle/_ref/{jacobi,gauss_seidel}.  The reference defines non-inline
// functions in headers, so the application, the library sources
// (interface.cpp, error_handler.cpp) and the Matrix Market reader (mmio.cpp)
// are compiled as ONE translation unit.  The printed iteration log of these
// programs is what tests/golden/make_solver_golden.py records as the golden
// output of the solver callers.

#include "interface.cpp"
#include "error_handler.cpp"
#include "mmio.cpp"

#include SMAX_APP_SOURCE
