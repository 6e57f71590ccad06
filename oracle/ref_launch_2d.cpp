// Launch wrappers around the reference's 2D barotropic kernels
// (modules/mod_cppkernels.cpp:12-250), host-compiled by oracle/build_ref.py.
// Test infrastructure only.  Each wrapper runs `n` CUDA threads of the kernel
// (n = grid * block of the reference's launch) through sfref_run.
#include "ref_host_shim.h"
#include SFREF_SOURCE

typedef const double* cdp;
extern "C" {
void sfref_initialize(long n, int omp, unsigned K, unsigned J, unsigned I,
                      double* on_u, double* om_v, double* pn, double* pm) {
    sfref_run(initialize, n, omp, K, J, I, on_u, om_v, pn, pm);
}
void sfref_computeMomentumRHSPred(long n, int omp, cdp h, cdp rhs_ubar, cdp rhs_vbar,
                                  cdp zeta_t0, cdp zeta_t2, double g, double weight) {
    sfref_run(computeMomentumRHSPred, n, omp, h, rhs_ubar, rhs_vbar, zeta_t0, zeta_t2, g, weight);
}
void sfref_computeMomentumRHSCorr(long n, int omp, cdp h, cdp rhs_ubar, cdp rhs_vbar,
                                  cdp zeta_t0, cdp zeta_t1, cdp zeta_t2, double g) {
    sfref_run(computeMomentumRHSCorr, n, omp, h, rhs_ubar, rhs_vbar, zeta_t0, zeta_t1, zeta_t2, g);
}
void sfref_computeZetaRHS(long n, int omp, cdp zeta, cdp h, double* ubar, cdp vbar, cdp DU_avg1,
                          cdp DV_avg1, cdp Zt_avg1, bool isPredictor, cdp weight1, cdp weight2,
                          int iif, double* res) {
    sfref_run(computeZetaRHS, n, omp, zeta, h, ubar, vbar, DU_avg1, DV_avg1, Zt_avg1, isPredictor,
              weight1, weight2, iif, res);
}
void sfref_computeZetaPred(long n, int omp, double Dt, cdp z0, cdp z1, cdp z2, cdp rz1) {
    sfref_run(computeZetaPred, n, omp, Dt, z0, z1, z2, rz1);
}
void sfref_computeMomentumPred(long n, int omp, double Dt, cdp u_t1, cdp u_t2, cdp v_t1, cdp v_t2,
                               cdp rhsu, cdp rhsv, cdp h, cdp zeta_t1, cdp zeta_t2) {
    sfref_run(computeMomentumPred, n, omp, Dt, u_t1, u_t2, v_t1, v_t2, rhsu, rhsv, h, zeta_t1, zeta_t2);
}
void sfref_AdamsMoultonCorr3rd(long n, int omp, double Dt, cdp v_t2, cdp r0, cdp r1, cdp r2) {
    sfref_run(AdamsMoultonCorr3rd, n, omp, Dt, v_t2, r0, r1, r2);
}
void sfref_AdamsMoultonCorr3rd2(long n, int omp, double Dt, cdp u_t2, cdp v_t2, cdp ru0, cdp ru1,
                                cdp ru2, cdp rv0, cdp rv1, cdp rv2, cdp h, cdp z1, cdp z2) {
    sfref_run(AdamsMoultonCorr3rd2, n, omp, Dt, u_t2, v_t2, ru0, ru1, ru2, rv0, rv1, rv2, h, z1, z2);
}
}
