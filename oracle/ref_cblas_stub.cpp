// TEST INFRASTRUCTURE ONLY. Link-time stub for the CBLAS call on the reference's unused host
// SPH path (src/compute_SPH.cpp:46-54), so that the reference CUDA library built by
// oracle/Makefile has no unresolved symbols.
#include <cstdio>
#include <cstdlib>
#include "cblas.h"
extern "C" {
void cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, double,
                 const double *, int, const double *, int, double, double *, int) {
   fprintf(stderr, "cblas_dgemm stub called\n");
   abort();
}

}
