// Aborting definitions for the distributed routines declared in
// pblas_decl.h (never reached on a 1x1 process grid).  Test infrastructure.
#include <cstdio>
#include <cstdlib>
#include "pblas_decl.h"
static void never(const char* f)
{ std::fprintf(stderr, "%s called on one process\n", f); std::abort(); }
extern "C" void pdgemm_(...) { never("pdgemm_"); }
extern "C" void pdgetrf_(...) { never("pdgetrf_"); }
extern "C" void pdgetri_(...) { never("pdgetri_"); }
extern "C" void pdlapv2_(...) { never("pdlapv2_"); }
extern "C" void pdpocon_(...) { never("pdpocon_"); }
extern "C" void pdpotrf_(...) { never("pdpotrf_"); }
extern "C" void pdpotri_(...) { never("pdpotri_"); }
extern "C" void pdsyev_(...) { never("pdsyev_"); }
extern "C" void pdsyevd_(...) { never("pdsyevd_"); }
extern "C" void pdsyevx_(...) { never("pdsyevx_"); }
extern "C" void pdsygst_(...) { never("pdsygst_"); }
extern "C" void pdsymm_(...) { never("pdsymm_"); }
extern "C" void pdsyrk_(...) { never("pdsyrk_"); }
extern "C" void pdtrmm_(...) { never("pdtrmm_"); }
extern "C" void pdtrsm_(...) { never("pdtrsm_"); }
extern "C" void pdtrtri_(...) { never("pdtrtri_"); }
extern "C" void pdtrtrs_(...) { never("pdtrtrs_"); }
extern "C" void pzgemm_(...) { never("pzgemm_"); }
extern "C" void pzgetrf_(...) { never("pzgetrf_"); }
extern "C" void pzgetri_(...) { never("pzgetri_"); }
extern "C" void pzheev_(...) { never("pzheev_"); }
extern "C" void pzheevd_(...) { never("pzheevd_"); }
extern "C" void pzhemm_(...) { never("pzhemm_"); }
extern "C" void pzherk_(...) { never("pzherk_"); }
extern "C" void pzlapv2_(...) { never("pzlapv2_"); }
extern "C" void pzpotrf_(...) { never("pzpotrf_"); }
extern "C" void pzsymm_(...) { never("pzsymm_"); }
extern "C" void pztrsm_(...) { never("pztrsm_"); }
extern "C" void pztrtri_(...) { never("pztrtri_"); }
extern "C" void pztrtrs_(...) { never("pztrtrs_"); }
extern "C" double pdlatra_(...) { never("pdlatra_"); return 0.0; }
