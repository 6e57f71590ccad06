// Launch wrappers around the reference's 3D momentum RHS kernels
// (nonlinear/rhs_kernels.cpp:7-224), host-compiled by oracle/build_ref.py.
// Test infrastructure only.
#include "ref_host_shim.h"
#include SFREF_SOURCE

typedef const double* cdp;
extern "C" {
void sfref_initialize(long n, int omp, unsigned K, unsigned J, unsigned I,
                      double* on_u, double* om_v, double* pn, double* pm) {
    sfref_run(initialize, n, omp, K, J, I, on_u, om_v, pn, pm);
}
void sfref_addCoriolis(long n, int omp, cdp fomn, cdp u, cdp v, cdp ru, cdp rv, cdp Hz) {
    sfref_run(addCoriolis, n, omp, fomn, u, v, ru, rv, Hz);
}
void sfref_horizontalAdvection(long n, int omp, cdp u, cdp v, cdp Huon, cdp Hvom, cdp ru, cdp rv,
                               const int* BC) {
    sfref_run(horizontalAdvection, n, omp, u, v, Huon, Hvom, ru, rv, BC);
}
void sfref_verticalAdvection(long n, int omp, cdp u, cdp v, cdp W, cdp ru, cdp rv, const int* BC) {
    sfref_run(verticalAdvection, n, omp, u, v, W, ru, rv, BC);
}
void sfref_vertIntegral(long n, int omp, cdp var, cdp sum) {
    sfref_run(vertIntegral, n, omp, var, sum);
}
}
