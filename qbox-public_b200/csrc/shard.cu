// Band pairs of one SlaterDet split over GPUs: the reference's state axis
// (nstb of MPIdata::set, src/MPIdata.cpp:55-121; the columns of c_,
// src/SlaterDet.cpp:84-93) for the FFT work of the electronic step.
//
// Every GPU holds the whole coefficient block; each one transforms a
// contiguous range of band pairs in update_density and in the local part of
// H*psi.  The partial densities are summed over the GPUs
// (src/ChargeDensity.cpp:166, MPI_Allreduce over the state communicator)
// and each GPU's H*psi bands are broadcast to the others, after which every
// GPU runs the same FP64/split-precision products, Cholesky and polar
// iteration on the same data (the library's kernels are deterministic), so
// the replicas stay identical without exchanging anything else.
//
// The collectives are NCCL's, over NVLink.  The library loads libnccl.so.2
// when a context is first sharded (no link-time dependency); the caller
// creates the group's unique id on one rank (qbx_nccl_unique_id) and hands
// it to every rank by its own means.
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/qbx.h"
#include "qbx_internal.h"

struct qbx_context;   // defined in capi.cu
namespace qbx {
Context& context_of(qbx_context* h);
}

namespace {

struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                             cudaStream_t) = nullptr;
  ncclResult_t (*broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*group_start)() = nullptr;
  ncclResult_t (*group_end)() = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};

const NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  static std::string fail;
  std::call_once(once, []() {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      fail = "libnccl.so.2 could not be loaded";
      return;
    }
    auto sym = [&](auto& fn, const char* name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
      if (!fn) fail = std::string("NCCL symbol missing: ") + name;
    };
    sym(api.get_unique_id, "ncclGetUniqueId");
    sym(api.comm_init_rank, "ncclCommInitRank");
    sym(api.comm_destroy, "ncclCommDestroy");
    sym(api.all_reduce, "ncclAllReduce");
    sym(api.broadcast, "ncclBroadcast");
    sym(api.group_start, "ncclGroupStart");
    sym(api.group_end, "ncclGroupEnd");
    sym(api.error_string, "ncclGetErrorString");
  });
  QBX_REQUIRE(fail.empty(), 70, fail);
  return api;
}

void nccl_check(ncclResult_t r, const char* what) {
  if (r != ncclSuccess)
    throw qbx::Error{71, std::string(what) + ": " + nccl().error_string(r)};
}

// pairs [lo, hi) of rank r among n: contiguous, sizes differing by one at most
void pair_range(int npairs, int r, int n, int& lo, int& hi) {
  lo = (int)((long long)npairs * r / n);
  hi = (int)((long long)npairs * (r + 1) / n);
}

}  // namespace

namespace qbx {

void shard_pairs(const Context& ctx, int& lo, int& hi) {
  pair_range((ctx.nst + 1) / 2, ctx.shard_rank, ctx.shard_n, lo, hi);
}

void shard_sum(Context& ctx, double* x, size_t n) {
  nccl_check(nccl().all_reduce(x, x, n, ncclDouble, ncclSum, (ncclComm_t)ctx.shard_comm,
                               ctx.stream),
             "ncclAllReduce of the density");
}

void shard_gather_bands(Context& ctx, double* x) {
  const size_t per_band = 2 * (size_t)ctx.wb.ng;
  const int npairs = (ctx.nst + 1) / 2;
  const NcclApi& api = nccl();
  nccl_check(api.group_start(), "ncclGroupStart");
  for (int r = 0; r < ctx.shard_n; r++) {
    int lo = 0, hi = 0;
    pair_range(npairs, r, ctx.shard_n, lo, hi);
    const int b0 = 2 * lo, b1 = std::min(2 * hi, ctx.nst);
    if (b1 <= b0) continue;
    double* blk = x + per_band * b0;
    const ncclResult_t e = api.broadcast(blk, blk, per_band * (b1 - b0), ncclDouble, r,
                                         (ncclComm_t)ctx.shard_comm, ctx.stream);
    if (e != ncclSuccess) {
      api.group_end();
      nccl_check(e, "ncclBroadcast of H*psi bands");
    }
  }
  nccl_check(api.group_end(), "ncclGroupEnd");
}

void shard_release(Context& ctx) {
  if (ctx.shard_comm) nccl().comm_destroy((ncclComm_t)ctx.shard_comm);
  ctx.shard_comm = nullptr;
  ctx.shard_rank = 0;
  ctx.shard_n = 1;
}

}  // namespace qbx

extern "C" {

int qbx_nccl_unique_id(unsigned char id[QBX_NCCL_ID_BYTES]) {
  if (!id) return 1;
  try {
    ncclUniqueId u;
    nccl_check(nccl().get_unique_id(&u), "ncclGetUniqueId");
    static_assert(sizeof(u) == QBX_NCCL_ID_BYTES, "NCCL unique id size");
    std::memcpy(id, &u, sizeof(u));
    return 0;
  } catch (const qbx::Error& e) {
    return e.code > 0 ? e.code : 1;
  }
}

int qbx_shard_pairs(int nst, int rank, int nranks, int* first_pair, int* end_pair) {
  if (nst < 1 || nranks < 1 || rank < 0 || rank >= nranks || !first_pair || !end_pair) return 1;
  pair_range((nst + 1) / 2, rank, nranks, *first_pair, *end_pair);
  return 0;
}

int qbx_set_band_shard(qbx_context* h, int rank, int nranks,
                       const unsigned char id[QBX_NCCL_ID_BYTES]) {
  if (!h) return 1;
  qbx::Context& c = qbx::context_of(h);
  try {
    QBX_CUDA(cudaSetDevice(c.device));
    QBX_REQUIRE(c.have_cell, 7, "qbx_set_cell has not been called");
    QBX_REQUIRE(nranks >= 1 && rank >= 0 && rank < nranks, 1, "bad rank or group size");
    QBX_REQUIRE(c.kpts.empty(), 1, "band sharding works on the Gamma SlaterDet");
    QBX_REQUIRE(!c.step_graph, 1, "band sharding and captured steps are exclusive");
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    qbx::shard_release(c);
    QBX_REQUIRE(nranks == 1 || id != nullptr, 1, "a group of several GPUs needs the NCCL unique id");
    if (id) {
      // a group of one GPU with an id also gets a communicator: the
      // collectives then run (trivially), as on several GPUs
      ncclUniqueId u;
      std::memcpy(&u, id, sizeof(u));
      ncclComm_t comm = nullptr;
      nccl_check(nccl().comm_init_rank(&comm, nranks, u, rank), "ncclCommInitRank");
      c.shard_comm = comm;
      c.shard_rank = rank;
      c.shard_n = nranks;
    }
    c.psir_valid = false;
    c.last_error.clear();
    return 0;
  } catch (const qbx::Error& e) {
    c.last_error = e.msg;
    return e.code > 0 ? e.code : 1;
  } catch (const std::exception& e) {
    c.last_error = e.what();
    return 6;
  }
}

}  // extern "C"
