// Launch wrappers around the reference's boundary scatter kernels
// (modules/mod_BC.c:6-23), host-compiled by oracle/build_ref.py.
// Test infrastructure only.
#include "ref_host_shim.h"
#include SFREF_SOURCE

extern "C" {
void sfref_setBC(long n, int omp, double* var, const int* idx, unsigned size, double val) {
    sfref_run(setBC, n, omp, var, idx, size, val);
}
void sfref_copyBC(long n, int omp, double* var, const unsigned* idx1, const unsigned* idx2,
                  unsigned size) {
    sfref_run(copyBC, n, omp, var, idx1, idx2, size);
}
}
