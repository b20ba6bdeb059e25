// Declarations of the distributed (PBLAS/ScaLAPACK) routines that the
// reference's Matrix.cpp names in branches taken only on process grids larger
// than 1x1.  The oracle runs on one process, so these are never called; the
// matching definitions in pblas_stub.cpp abort.  Test infrastructure only.
#ifndef QBX_ORACLE_PBLAS_DECL_H
#define QBX_ORACLE_PBLAS_DECL_H
extern "C" {
void pdgemm_(...);
void pdgetrf_(...);
void pdgetri_(...);
void pdlapv2_(...);
void pdpocon_(...);
void pdpotrf_(...);
void pdpotri_(...);
void pdsyev_(...);
void pdsyevd_(...);
void pdsyevx_(...);
void pdsygst_(...);
void pdsymm_(...);
void pdsyrk_(...);
void pdtrmm_(...);
void pdtrsm_(...);
void pdtrtri_(...);
void pdtrtrs_(...);
void pzgemm_(...);
void pzgetrf_(...);
void pzgetri_(...);
void pzheev_(...);
void pzheevd_(...);
void pzhemm_(...);
void pzherk_(...);
void pzlapv2_(...);
void pzpotrf_(...);
void pzsymm_(...);
void pztrsm_(...);
void pztrtri_(...);
void pztrtrs_(...);
double pdlatra_(...);
}
#endif
