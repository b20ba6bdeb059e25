// One-process BLACS for compiling the reference Qbox sources as the CPU oracle
// (oracle/_ref).  Test infrastructure, not product.
//
// The reference declares these functions in src/blacs.h:48-73 and calls them
// from src/Context.cpp:31-345.  Without SCALAPACK they have C++ linkage, so
// this file includes the reference header to get identical signatures.  With
// one process every grid is 1x1, every sum/max/min/broadcast is the identity
// and point-to-point sends never happen.
#include <cstdio>
#include <cstdlib>
#include "blacs.h"

static void one_proc_only(const char* f)
{
  std::fprintf(stderr, "BLACS stub: %s needs more than one process\n", f);
  std::abort();
}

void Cblacs_pinfo(int* mypnum, int* nprocs) { *mypnum = 0; *nprocs = 1; }
void Cblacs_get(int, int, int* val) { *val = 0; }
int Csys2blacs_handle(MPI_Comm) { return 0; }
void Cblacs_barrier(int, const char*) {}
void Cblacs_gridinfo(int ictxt, int* nprow, int* npcol, int* myrow, int* mycol)
{
  if ( ictxt < 0 ) { *nprow = *npcol = *myrow = *mycol = -1; return; }
  *nprow = 1; *npcol = 1; *myrow = 0; *mycol = 0;
}
void Cblacs_gridinit(int* ictxt, char[], int nprow, int npcol)
{
  if ( nprow * npcol != 1 ) one_proc_only("Cblacs_gridinit");
  *ictxt = 0;
}
void Cblacs_gridmap(int* ictxt, int*, int, int nprow, int npcol)
{
  if ( nprow * npcol != 1 ) one_proc_only("Cblacs_gridmap");
  *ictxt = 0;
}
void Cblacs_abort(int, int code) { std::exit(code); }
void Cblacs_gridexit(int) {}
int Cblacs_pnum(int, int, int) { return 0; }

void Cdgesd2d(int, int, int, double*, int, int, int)
{ one_proc_only("Cdgesd2d"); }
void Cdgerv2d(int, int, int, double*, int, int, int)
{ one_proc_only("Cdgerv2d"); }
void Cdgsum2d(int, char*, char*, int, int, double*, int, int, int) {}
void Cdgamx2d(int, char*, char*, int m, int n, double*, int, int* ra, int* ca,
  int rcflag, int, int)
{
  if ( rcflag != -1 && ra && ca )
    for ( int i = 0; i < m * n; i++ ) { ra[i] = 0; ca[i] = 0; }
}
void Cdgamn2d(int, char*, char*, int m, int n, double*, int, int* ra, int* ca,
  int rcflag, int, int)
{
  if ( rcflag != -1 && ra && ca )
    for ( int i = 0; i < m * n; i++ ) { ra[i] = 0; ca[i] = 0; }
}
void Cdgebs2d(int, char*, char*, int, int, double*, int) {}
void Cdgebr2d(int, char*, char*, int, int, double*, int, int, int) {}
void Cigesd2d(int, int, int, int*, int, int, int)
{ one_proc_only("Cigesd2d"); }
void Cigerv2d(int, int, int, int*, int, int, int)
{ one_proc_only("Cigerv2d"); }
void Cigsum2d(int, char*, char*, int, int, int*, int, int, int) {}
void Cigamx2d(int, char*, char*, int m, int n, int*, int, int* ra, int* ca,
  int rcflag, int, int)
{
  if ( rcflag != -1 && ra && ca )
    for ( int i = 0; i < m * n; i++ ) { ra[i] = 0; ca[i] = 0; }
}
void Cigamn2d(int, char*, char*, int m, int n, int*, int, int* ra, int* ca,
  int rcflag, int, int)
{
  if ( rcflag != -1 && ra && ca )
    for ( int i = 0; i < m * n; i++ ) { ra[i] = 0; ca[i] = 0; }
}
void Cigebs2d(int, char*, char*, int, int, int*, int) {}
void Cigebr2d(int, char*, char*, int, int, int*, int, int, int) {}

// ScaLAPACK's NUMROC tool function (number of rows or columns of a
// block-cyclically distributed matrix owned by process iproc).  Matrix.cpp
// calls it unconditionally; the formula is ScaLAPACK's published one.
extern "C" int numroc_(const int* n, const int* nb, const int* iproc,
  const int* isrcproc, const int* nprocs)
{
  const int mydist = ( *nprocs + *iproc - *isrcproc ) % *nprocs;
  const int nblocks = *n / *nb;
  int num = ( nblocks / *nprocs ) * *nb;
  const int extrablks = nblocks % *nprocs;
  if ( mydist < extrablks ) num += *nb;
  else if ( mydist == extrablks ) num += *n % *nb;
  return num;
}
