// Single-rank stand-in for <mpi.h>, used only to compile the reference Qbox
// sources as the CPU oracle (oracle/_ref).  Test infrastructure, not product.
//
// Every communicator has exactly one rank (rank 0, size 1).  Reductions,
// broadcasts and all-to-all exchanges therefore reduce to local copies.
// The reference needs these calls even at one task: MPIdata::set builds a
// 4-D Cartesian communicator (src/MPIdata.cpp:55-120), BasisMapping uses
// Alltoallv only when nprocs > 1 (src/BasisMapping.cpp:445-540).
#ifndef QBX_ORACLE_SHIM_MPI_H
#define QBX_ORACLE_SHIM_MPI_H

#include <cstring>
#include <cstdlib>
#include <cstdio>
#include <sys/time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;   // value = size of one element in bytes
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_SUCCESS 0
#define MPI_CHAR 1
#define MPI_BYTE 1
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_LONG 8
#define MPI_LONG_LONG 8
#define MPI_DOUBLE 8
#define MPI_DOUBLE_COMPLEX 16
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_INFO_NULL 0
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_IN_PLACE ((void*)1)

static inline void qbx_mpi_copy(const void* s, void* r, int n, MPI_Datatype t)
{
  if ( s != MPI_IN_PLACE && s != r && n > 0 )
    std::memmove(r, s, (size_t) n * (size_t) t);
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code)
{ std::fprintf(stderr, "MPI_Abort(%d)\n", code); std::exit(code); return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* d) { *d = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm*) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int,
  MPI_Comm* c) { *c = MPI_COMM_WORLD; return 0; }
static inline int MPI_Cart_sub(MPI_Comm, const int*, MPI_Comm* c)
{ *c = MPI_COMM_WORLD; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int n, int* coords)
{ for ( int i = 0; i < n; i++ ) coords[i] = 0; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t,
  MPI_Op, MPI_Comm) { qbx_mpi_copy(s, r, n, t); return 0; }
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t,
  MPI_Op, int, MPI_Comm) { qbx_mpi_copy(s, r, n, t); return 0; }
static inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t,
  MPI_Op, MPI_Comm) { qbx_mpi_copy(s, r, n, t); return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm)
{ return 0; }
static inline int MPI_Alltoall(const void* s, int sc, MPI_Datatype st, void* r,
  int, MPI_Datatype, MPI_Comm) { qbx_mpi_copy(s, r, sc, st); return 0; }
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd,
  MPI_Datatype st, void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm)
{
  std::memmove((char*) r + (size_t) rd[0] * st,
               (const char*) s + (size_t) sd[0] * st, (size_t) sc[0] * st);
  return 0;
}
static inline int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r,
  int, MPI_Datatype, MPI_Comm) { qbx_mpi_copy(s, r, sc, st); return 0; }
static inline int MPI_Allgatherv(const void* s, int sc, MPI_Datatype st,
  void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm)
{ qbx_mpi_copy(s, (char*) r + (size_t) rd[0] * st, sc, st); return 0; }
static inline int MPI_Gatherv(const void* s, int sc, MPI_Datatype st, void* r,
  const int*, const int* rd, MPI_Datatype, int, MPI_Comm)
{ qbx_mpi_copy(s, (char*) r + (size_t) rd[0] * st, sc, st); return 0; }
static inline int MPI_Scatterv(const void* s, const int* sc, const int* sd,
  MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm)
{ qbx_mpi_copy((const char*) s + (size_t) sd[0] * st, r, sc[0], st); return 0; }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm)
{ std::fprintf(stderr, "MPI_Send on one rank\n"); std::abort(); return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm,
  MPI_Status*)
{ std::fprintf(stderr, "MPI_Recv on one rank\n"); std::abort(); return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm,
  MPI_Request*) { std::abort(); return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm,
  MPI_Request*) { std::abort(); return 0; }
static inline int MPI_Send_init(const void*, int, MPI_Datatype, int, int,
  MPI_Comm, MPI_Request*) { return 0; }
static inline int MPI_Recv_init(void*, int, MPI_Datatype, int, int, MPI_Comm,
  MPI_Request*) { return 0; }
static inline int MPI_Start(MPI_Request*) { return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Request_free(MPI_Request*) { return 0; }
static inline int MPI_Get_count(const MPI_Status* s, MPI_Datatype, int* c)
{ *c = s ? s->count : 0; return 0; }
static inline int MPI_Get_processor_name(char* name, int* len)
{ std::strcpy(name, "localhost"); *len = 9; return 0; }
static inline double MPI_Wtime(void)
{ struct timeval tv; gettimeofday(&tv, 0); return tv.tv_sec + 1e-6 * tv.tv_usec; }
static inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File*)
{ std::abort(); return 0; }
static inline int MPI_File_close(MPI_File*) { return 0; }
static inline int MPI_File_set_size(MPI_File, MPI_Offset) { return 0; }
static inline int MPI_File_write(MPI_File, const void*, int, MPI_Datatype,
  MPI_Status*) { return 0; }
static inline int MPI_File_write_at(MPI_File, MPI_Offset, const void*, int,
  MPI_Datatype, MPI_Status*) { return 0; }
static inline int MPI_File_write_at_all(MPI_File, MPI_Offset, const void*, int,
  MPI_Datatype, MPI_Status*) { return 0; }

#endif
