// DTRTRS and ZTRTRS for the oracle build.  The OpenBLAS 0.3.15 library in the Python
// environment rejects DIAG='n' in its own DTRTRS ("parameter number 3 had an
// illegal value") when called from the reference's Matrix::trtrs
// (src/Matrix.cpp:1959-1989).  LAPACK defines DTRTRS as a singularity check
// on the diagonal followed by DTRSM, which is what this does; defining it in
// the executable takes precedence over the shared library's symbol.
// Test infrastructure, not product.
extern "C" void dtrsm_(const char*, const char*, const char*, const char*,
  const int*, const int*, const double*, const double*, const int*, double*,
  const int*);

extern "C" void dtrtrs_(const char* uplo, const char* trans, const char* diag,
  const int* n, const int* nrhs, const double* a, const int* lda, double* b,
  const int* ldb, int* info)
{
  *info = 0;
  if ( *n == 0 ) return;
  const bool unit = ( *diag == 'U' || *diag == 'u' );
  if ( !unit )
    for ( int i = 0; i < *n; i++ )
      if ( a[i + (long)i * *lda] == 0.0 ) { *info = i + 1; return; }
  const double one = 1.0;
  dtrsm_("L", uplo, trans, diag, n, nrhs, &one, a, lda, b, ldb);
}

// ZTRTRS, the same definition for complex matrices (ComplexMatrix::trtrs,
// src/Matrix.cpp:1997-2027, used by the complex-basis SlaterDet::ortho_align).
#include <complex>
extern "C" void ztrsm_(const char*, const char*, const char*, const char*,
  const int*, const int*, const std::complex<double>*, const std::complex<double>*,
  const int*, std::complex<double>*, const int*);

extern "C" void ztrtrs_(const char* uplo, const char* trans, const char* diag,
  const int* n, const int* nrhs, const std::complex<double>* a, const int* lda,
  std::complex<double>* b, const int* ldb, int* info)
{
  *info = 0;
  if ( *n == 0 ) return;
  const bool unit = ( *diag == 'U' || *diag == 'u' );
  if ( !unit )
    for ( int i = 0; i < *n; i++ )
      if ( a[i + (long)i * *lda] == 0.0 ) { *info = i + 1; return; }
  const std::complex<double> one = 1.0;
  ztrsm_("L", uplo, trans, diag, n, nrhs, &one, a, lda, b, ldb);
}
