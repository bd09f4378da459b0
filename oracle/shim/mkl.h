/* Stand-in for Intel MKL's mkl.h, which is not installed on this machine.
 * Test infrastructure only: lets the reference's solver_pardiso.cpp compile so
 * that its other translation units link.  PARDISO always reports error -1, so
 * the reference's "Pardiso_class"/"Pardiso_func" paths are unavailable; the
 * oracle uses the reference's "SuperLU_func" path instead. */
#ifndef OFEA_SHIM_MKL_H
#define OFEA_SHIM_MKL_H
typedef int MKL_INT;
static inline void PARDISO(void *pt, const MKL_INT *maxfct, const MKL_INT *mnum,
                           const MKL_INT *mtype, const MKL_INT *phase, const MKL_INT *n,
                           const void *a, const MKL_INT *ia, const MKL_INT *ja,
                           MKL_INT *perm, const MKL_INT *nrhs, MKL_INT *iparm,
                           const MKL_INT *msglvl, void *b, void *x, MKL_INT *error)
{
    (void)pt; (void)maxfct; (void)mnum; (void)mtype; (void)phase; (void)n; (void)a;
    (void)ia; (void)ja; (void)perm; (void)nrhs; (void)iparm; (void)msglvl; (void)b; (void)x;
    *error = -1;
}
#endif
