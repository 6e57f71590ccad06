// Launch wrappers around the reference's 3D step kernels
// (nonlinear/step3D_uv.kernels.cpp:21-739), host-compiled by oracle/build_ref.py.
// Test infrastructure only.
#include "ref_host_shim.h"
#include SFREF_SOURCE

typedef const double* cdp;
extern "C" {
void sfref_initialize(long n, int omp, unsigned K, unsigned J, unsigned I,
                      double* on_u, double* om_v, double* pn, double* pm) {
    sfref_run(initialize, n, omp, K, J, I, on_u, om_v, pn, pm);
}
void sfref_setVerticalVelEq(long n, int omp, double* SD, double* D, double* RHS) {
    sfref_run(setVerticalVelEq, n, omp, SD, D, RHS);
}
void sfref_omega(long n, int omp, cdp W, cdp u, cdp v, cdp Huon, cdp Hvom, cdp z_w, const int* BC) {
    sfref_run(omega, n, omp, W, u, v, Huon, Hvom, z_w, BC);
}
void sfref_set_depth(long n, int omp, int Vtransform, cdp Zt_avg1, cdp z_w, cdp z_r, cdp h, double hc,
                     cdp Hz, cdp sc_r, cdp sc_w, cdp Cs_r, cdp Cs_w) {
    sfref_run(set_depth, n, omp, Vtransform, Zt_avg1, z_w, z_r, h, hc, Hz, sc_r, sc_w, Cs_r, Cs_w);
}
void sfref_set_zeta(long n, int omp, cdp zeta1, cdp zeta2, cdp Zt_avg1) {
    sfref_run(set_zeta, n, omp, zeta1, zeta2, Zt_avg1);
}
void sfref_setLateralUVBCs(long n, int omp, double t, double* u, double* v, const int* uIdx2,
                           const int* vIdx2, const int* uType, const int* vType) {
    sfref_run(setLateralUVBCs, n, omp, t, u, v, uIdx2, vIdx2, uType, vType);
}
void sfref_set_maxflux(long n, int omp, cdp u, cdp v, cdp Huon, cdp Hvom, cdp Hz) {
    sfref_run(set_maxflux, n, omp, u, v, Huon, Hvom, Hz);
}
void sfref_step3d_UV(long n, int omp, double* u, double* v, cdp ru, cdp rv, cdp ubar_t1, cdp vbar_t1,
                     cdp ubar_t2, cdp vbar_t2, cdp Hz, cdp Akv, cdp z_r, cdp DU_avg1, cdp DV_avg1,
                     cdp tmpU, cdp tmpV, cdp h, int iic, int ntfirst, double lambda, double AK,
                     double Dt) {
    sfref_run(step3d_UV, n, omp, u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, Akv, z_r,
              DU_avg1, DV_avg1, tmpU, tmpV, h, iic, ntfirst, lambda, AK, Dt);
}
}
