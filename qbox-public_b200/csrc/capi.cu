// C ABI of the library (declared in include/qbx.h).  Each entry point wraps
// one operation of the reference's class API on the electronic-step path,
// converts exceptions to status codes and keeps the message for
// qbx_last_error().
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <new>
#include <stdexcept>
#include <thread>
#include <atomic>
#include <tuple>

#include "../../include/qbx.h"
#include "qbx_internal.h"

struct qbx_context {
  qbx::Context c;
  std::vector<int> perm;          // caller row -> internal row
  int* d_perm = nullptr;
};

using namespace qbx;

namespace {

template <typename F>
int guarded(qbx_context* h, F f) {
  if (!h) return 1;
  try {
    QBX_CUDA(cudaSetDevice(h->c.device));
    f(h->c);
    h->c.last_error.clear();
    return 0;
  } catch (const Error& e) {
    h->c.last_error = e.msg;
    return e.code > 0 ? e.code : 1;
  } catch (const std::bad_alloc&) {
    h->c.last_error = "host allocation failed";
    return 5;
  } catch (const std::exception& e) {
    h->c.last_error = e.what();
    return 6;
  }
}

// Captured steps hold the buffer pointers and launch shapes of the moment of
// capture; anything that changes those drops them.
void drop_batch(Context& c) {
  if (c.batch.exec) cudaGraphExecDestroy(c.batch.exec);
  c.batch = BatchGraph{};
}

void drop_graphs(Context& c) {
  for (auto& g : c.graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = StepGraph{};
  }
  drop_batch(c);
}

void free_cell(Context& c) {
  drop_graphs(c);
  free_kpoints(c);
  if (c.s_in) cudaStreamSynchronize(c.s_in);
  if (c.s_out) cudaStreamSynchronize(c.s_out);
  dfree(c.d_cin);
  dfree(c.d_cout);
  if (c.d_psir) { cudaFree(c.d_psir); c.d_psir = nullptr; }
  c.psir_bytes = 0;
  c.psir_valid = false;
  c.in_pending = c.finish_pending = false;
  free_mixed(c);
  free_mix(c);
  if (c.have_wgrid) free_sticks(c.dwg);
  c.have_wgrid = false;
  free_sticks(c.dws);
  free_sticks(c.dvs);
  double** bufs[] = {&c.d_gx_w, &c.d_g2_w, &c.d_gx_v, &c.d_g2i_v, &c.d_c, &c.d_hc, &c.d_c_last,
                     &c.d_dc_last, &c.d_ctmp, &c.d_occ, &c.d_rhor, &c.d_vr, &c.d_vxc,
                     &c.d_exc, &c.d_vx2, &c.d_grad, &c.d_rhog, &c.d_vion, &c.d_rhops,
                     &c.d_vtmp_g, &c.d_vtmp_g2, &c.d_xc_g, &c.d_nn, &c.d_nn2, &c.d_nn3, &c.d_nn4, &c.d_nn5,
                     &c.d_solver_work, &c.d_red, &c.d_scalars, &c.d_prec, &c.d_jd_h,
                     &c.d_jd_w, &c.d_jd_work, &c.d_wfv, &c.d_xsd, &c.d_xgrid};
  for (double** b : bufs) dfree(*b);
  dfree(c.d_ipiv);
  dfree(c.d_info);
  if (c.d_grid) { cudaFree(c.d_grid); c.d_grid = nullptr; }
  if (c.d_zbuf) { cudaFree(c.d_zbuf); c.d_zbuf = nullptr; }
  if (c.d_zfast) { cudaFree(c.d_zfast); c.d_zfast = nullptr; }
  dfree(c.d_vr32);
  c.have_cell = false;
}

void free_atoms(Context& c) {
  drop_graphs(c);
  kpoints_atoms_changed(c);
  if (c.h_fion) { cudaFreeHost(c.h_fion); c.h_fion = nullptr; }
  double** bufs[] = {&c.d_anl, &c.d_fnl, &c.d_dfnl, &c.d_pdfac, &c.d_sfac, &c.d_vps,
                     &c.d_rhops_sp, &c.d_fion, &c.d_dvps, &c.d_vnl, &c.d_dvnl,
                     &c.d_tau_all, &c.d_astress, &c.d_twnl, &c.d_phase_tab, &c.d_fpart};
  for (double** b : bufs) dfree(*b);
  c.phase_tab_bytes = 0;
  c.fpart_elems = 0;
  dfree(c.d_patom);
  dfree(c.d_pcol);
  if (c.sa_hi) { cudaFree(c.sa_hi); c.sa_hi = nullptr; }
  if (c.sa_lo) { cudaFree(c.sa_lo); c.sa_lo = nullptr; }
  c.have_stress = false;
  c.nproj = 0;
}

void fill_energies(const Context& c, double* e) {
  if (!e) return;
  const double v[QBX_NENERGY] = {c.ekin, c.eps, c.enl, c.ehart, c.ecoul, c.exc, c.esr, c.eself,
                                 c.etotal, c.eigsum, c.total_charge, c.theta};
  std::memcpy(e, v, sizeof(v));
}

__global__ void k_permute(const double2* __restrict__ in, const int* __restrict__ perm, int ngw,
                          int nst, int to_internal, double2* __restrict__ out) {
  const size_t n = (size_t)ngw * nst;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t b = t / ngw;
    const int i = (int)(t - b * ngw);
    if (to_internal) out[b * ngw + perm[i]] = in[t];
    else out[t] = in[b * ngw + perm[i]];
  }
}

// density weights occ/Omega are kept in d_wdens (a slice of the scalar pool)
void upload_weights(Context& c) {
  std::vector<double> w(c.nst);
  for (int n = 0; n < c.nst; n++) w[n] = c.occ[n] / c.wb.omega;
  h2d_sync(c.d_scalars + kSlots, w.data(), sizeof(double) * c.nst);
}

void check_ready(const Context& c, bool atoms) {
  QBX_REQUIRE(c.have_cell, 7, "qbx_set_cell has not been called");
  if (atoms) QBX_REQUIRE(c.d_vion != nullptr && !c.tau.empty(), 7, "qbx_set_atoms has not been called");
}

}  // namespace

// density weights live after the scalar slots
namespace qbx {
double* density_weights(Context& c) { return c.d_scalars + kSlots; }
Context& context_of(qbx_context* h) { return h->c; }
}

namespace {

// The energies, eigenvalue sum and forces of a step from the read-back slots.
void finish_step(Context& c, bool want_f, bool want_s) {
  finish_density(c);
  finish_vhxc(c);
  finish_energy(c, want_f);
  finish_eigsum(c);
  if (want_s) finish_stress(c);
}

// BOSampleStepper's electronic step (src/BOSampleStepper.cpp:795-1114 with
// nite = 0), every operation on c.stream.
void step_eager(Context& c, bool want_f, bool want_s, double* energies, double* fion) {
  if (!c.kpts.empty()) {
    // k points off Gamma: the same sequence on the complex SlaterDets
    QBX_REQUIRE(!want_f && !want_s, 1, "forces and stress are not available at k points off Gamma");
    update_density_k(c);
    update_vhxc(c);
    energy_k(c, true);
    eigsum_k(c);
    readback(c, false);
    check_status(c);
    finish_step(c, false, false);
    fill_energies(c, energies);
    psda_update_k(c);
    readback(c, false);
    check_status(c);
    finish_theta(c);
    return;
  }
  // psi(r) of the density pass is reused by the H*psi pass
  c.psir_store = true;
  update_density(c);
  c.psir_store = false;
  update_vhxc(c);
  c.psir_use = true;
  energy(c, true, want_f);
  c.psir_use = false;
  c.psir_valid = false;
  if (want_s) compute_stress(c);
  launch_eigsum(c);
  readback(c, want_f);
  check_status(c);
  finish_step(c, want_f, want_s);
  fill_energies(c, energies);
  if (want_f && fion) std::memcpy(fion, c.fion.data(), sizeof(double) * c.fion.size());
  if (c.wf_dyn == 1) jd_update(c);
  else psda_update(c, PSDA_PREC_FROM_ENERGY);   // energy() ran on this C
  readback(c, false);
  check_status(c);
  finish_theta(c);
}

// The same PSDA step captured into one graph: the reductions stay on the
// device, the Anderson theta and the polar iteration are decided there
// (conditional nodes), and the last nodes copy slots, status and forces to
// the pinned mirrors.  The graph is instantiated, not launched.
// The operations of one PSDA step on c.stream while that stream is being
// captured (it may be one branch of a larger capture).  Host state the
// recording changes (profiling, the extrapolation flag, the launch count) is
// put back afterwards; returns the number of this library's kernels recorded.
long record_step(Context& c, bool want_f) {
  const bool prof = c.prof.on, extrap = c.extrapolate, kextrap = c.kpts_extrapolate;
  const long n0 = c.nlaunch;
  c.prof.on = false;
  c.capturing = true;
  auto restore = [&]() {
    c.psir_store = c.psir_use = c.psir_valid = false;
    c.capturing = false;
    c.prof.on = prof;
    c.extrapolate = extrap;
    c.kpts_extrapolate = kextrap;
  };
  try {
    if (!c.kpts.empty()) {
      // k points off Gamma: the same sequence on the complex SlaterDets
      update_density_k(c);
      update_vhxc(c);
      energy_k(c, true);
      eigsum_k(c);
      psda_update_k(c);
      enqueue_readback(c, false);
      restore();
      const long k = c.nlaunch - n0;
      c.nlaunch = n0;
      return k;
    }
    c.psir_store = true;
    update_density(c);
    c.psir_store = false;
    update_vhxc(c);
    c.psir_use = true;
    energy(c, true, want_f);
    c.psir_use = false;
    c.psir_valid = false;
    psda_update(c, PSDA_PREC_FROM_ENERGY | PSDA_EIGSUM);
    enqueue_readback(c, want_f);
  } catch (...) {
    restore();
    c.nlaunch = n0;
    throw;
  }
  restore();
  const long k = c.nlaunch - n0;
  c.nlaunch = n0;
  return k;
}

void capture_step(Context& c, bool want_f, StepGraph& g) {
  QBX_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
  cudaGraph_t graph = nullptr;
  try {
    g.nkernels = record_step(c, want_f);
  } catch (...) {
    cudaStreamEndCapture(c.stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  QBX_CUDA(cudaStreamEndCapture(c.stream, &graph));
  static std::atomic<long> next_id{1};
  g.id = next_id.fetch_add(1);
  cudaGraphInstantiateParams ip = {};
  const cudaError_t e = cudaGraphInstantiateWithParams(&g.exec, graph, &ip);
  if (e != cudaSuccess) {
    g.exec = nullptr;
    std::string why = std::string("graph instantiation: ") + cudaGetErrorString(e) +
                      " (result " + std::to_string((int)ip.result_out) + ")";
    if (ip.errNode_out) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(ip.errNode_out, &t) == cudaSuccess) {
        why += ", node type " + std::to_string((int)t);
        if (t == cudaGraphNodeTypeKernel) {
          cudaKernelNodeParams kp = {};
          const char* name = nullptr;
          if (cudaGraphKernelNodeGetParams(ip.errNode_out, &kp) == cudaSuccess &&
              cudaFuncGetName(&name, kp.func) == cudaSuccess && name)
            why += std::string(" ") + name;
        } else if (t == cudaGraphNodeTypeMemcpy) {
          cudaMemcpy3DParms mp = {};
          if (cudaGraphMemcpyNodeGetParams(ip.errNode_out, &mp) == cudaSuccess)
            why += ", copy kind " + std::to_string((int)mp.kind);
        }
      }
    }
    cudaGetLastError();
    cudaGraphDestroy(graph);
    g.id = 0;
    throw Error{57, why};
  }
  cudaGraphDestroy(graph);
}

// The captured graph of this step's configuration, or null when the step
// runs eagerly (graphs off, JD, stress, profiling, or the first use of the
// configuration, which sizes the lazily grown buffers before any capture).
StepGraph* step_graph_for(Context& c, bool want_f, bool want_s) {
  if (!c.step_graph || c.wf_dyn != 0 || want_s || c.prof.on) return nullptr;
  if (!c.kpts.empty() && want_f) return nullptr;
  const bool extrap = c.kpts.empty() ? c.extrapolate : c.kpts_extrapolate;
  StepGraph& g = c.graphs[(extrap ? 1 : 0) + (want_f ? 2 : 0)];
  if (g.exec) return &g;
  if (g.uses++ == 0) return nullptr;
  try {
    capture_step(c, want_f, g);
  } catch (const Error& e) {
    // a step that cannot be captured keeps running eagerly
    c.graph_note = e.msg;
    c.step_graph = false;
    return nullptr;
  }
  return &g;
}

void launch_step_graph(Context& c, StepGraph& g) {
  QBX_CUDA(cudaGraphLaunch(g.exec, c.stream));
  c.nlaunch += g.nkernels;
  c.graph_launches++;
}

// after the graph of a step has completed
// after the graph of a step has completed; the energies report the theta of
// the previous update, as the eager step (which reports before updating) does
void finish_graph_step(Context& c, bool want_f, double* energies, double* fion) {
  check_status(c);
  finish_step(c, want_f, false);
  fill_energies(c, energies);
  finish_theta(c);
  if (c.kpts.empty()) c.extrapolate = true;
  else c.kpts_extrapolate = true;
  if (want_f && fion) std::memcpy(fion, c.fion.data(), sizeof(double) * c.fion.size());
}

}  // namespace

extern "C" {

int qbx_version(void) { return 1; }

int qbx_create(qbx_context** out, int device, int precision) {
  if (!out) return 1;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return 8;
  if (device < 0 || device >= ndev) return 9;
  if (precision != QBX_FP64 && precision != QBX_MIXED) return 1;
  qbx_context* h = new (std::nothrow) qbx_context();
  if (!h) return 5;
  h->c.device = device;
  h->c.precision = precision;
  if (const char* e = std::getenv("QBX_GEMM_BACKEND")) h->c.gemm_backend = std::atoi(e) == 0 ? 0 : 1;
  // tall updates: the rotation of C uses TF32 splits (BF16 splits would
  // leave C orthonormal only to ~1e-5); the H*C updates use BF16 splits,
  // ~20% faster, whose ~1e-5 relative error only enters the step direction
  if (const char* e = std::getenv("QBX_TALL_KIND")) h->c.tall_kind = std::atoi(e) == 0 ? 0 : 1;
  if (const char* e = std::getenv("QBX_TC_CHUNK")) h->c.tc_chunk = std::max(1, std::min(64, std::atoi(e)));
  if (const char* e = std::getenv("QBX_TC_EPW")) h->c.tc_epw = std::atoi(e) == 4 ? 4 : 8;
  if (const char* e = std::getenv("QBX_TC_PAIR")) h->c.tc_pair = std::max(0, std::min(2, std::atoi(e)));
  if (const char* e = std::getenv("QBX_TC_PAIR_EPW")) h->c.tc_pair_epw = std::atoi(e) == 8 ? 8 : 16;
  if (const char* e = std::getenv("QBX_TC_TF32_MN")) h->c.tc_tf32_mn = std::atoi(e) != 0 ? 1 : 0;
  if (const char* e = std::getenv("QBX_STEP_FUSE")) h->c.step_fuse = std::atoi(e) != 0 ? 1 : 0;
  if (const char* e = std::getenv("QBX_TC_CORR_MUL")) h->c.tc_corr_mul = std::max(0, std::min(64, std::atoi(e)));
  if (const char* e = std::getenv("QBX_TALL_KIND_HC")) h->c.tall_kind_hc = std::atoi(e) == 1 ? 1 : 0;
  // batches of captured steps: one graph launch per context on its own
  // stream (default; 9.8 ms for 32 small systems) or one graph with every
  // context as a branch (15.7 ms: its conditional nodes serialise branches)
  if (const char* e = std::getenv("QBX_BATCH_GRAPH")) h->c.batch_single_graph = std::atoi(e) != 0;
  const int rc = guarded(h, [&](Context& c) {
    QBX_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    QBX_BLAS(cublasCreate(&c.blas));
    QBX_BLAS(cublasSetStream(c.blas, c.stream));
    QBX_SOLVER(cusolverDnCreate(&c.solver));
    for (auto& s : c.side) QBX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    // cuBLAS workspace owned by the context (rebound with every stream)
    c.blas_ws_bytes = (size_t)32 << 20;
    QBX_CUDA(cudaMalloc(&c.d_blas_ws, c.blas_ws_bytes));
    bind_stream(c, c.stream);
    // status words and the pinned mirrors of slots and status
    c.d_status = dalloc<int>(kStatus);
    QBX_CUDA(cudaMemset(c.d_status, 0, kStatus * sizeof(int)));
    QBX_CUDA(cudaMallocHost(&c.h_scalars, kSlots * sizeof(double)));
    QBX_CUDA(cudaMallocHost(&c.h_status, kStatus * sizeof(int)));
    std::memset(c.h_scalars, 0, kSlots * sizeof(double));
    std::memset(c.h_status, 0, kStatus * sizeof(int));
    QBX_CUDA(cudaDeviceSynchronize());
  });
  if (rc) { delete h; return rc; }
  *out = h;
  return 0;
}

void qbx_destroy(qbx_context* h) {
  if (!h) return;
  cudaSetDevice(h->c.device);
  if (h->c.stream) cudaStreamSynchronize(h->c.stream);
  try {
    shard_release(h->c);
  } catch (...) {
  }
  free_atoms(h->c);
  free_cell(h->c);
  dfree(h->d_perm);
  dfree(h->c.d_status);
  if (h->c.d_blas_ws) cudaFree(h->c.d_blas_ws);
  if (h->c.h_scalars) cudaFreeHost(h->c.h_scalars);
  if (h->c.h_status) cudaFreeHost(h->c.h_status);
  if (h->c.blas) cublasDestroy(h->c.blas);
  if (h->c.solver) cusolverDnDestroy(h->c.solver);
  for (auto s : h->c.side)
    if (s) cudaStreamDestroy(s);
  for (cudaStream_t s : {h->c.s_in, h->c.s_out})
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : {h->c.ev_in, h->c.ev_cin_free, h->c.ev_step, h->c.ev_out})
    if (e) cudaEventDestroy(e);
  if (h->c.stream) cudaStreamDestroy(h->c.stream);
  delete h;
}

const char* qbx_last_error(const qbx_context* h) {
  return h ? h->c.last_error.c_str() : "null context";
}

int qbx_set_precision(qbx_context* h, int precision) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(precision == QBX_FP64 || precision == QBX_MIXED, 1, "unknown precision");
    if (c.have_cell && precision != c.precision) {
      // the stick buffer holds the precision's complex type
      c.precision = precision;
      const size_t per_pair = (size_t)c.wb.n2 * c.wb.nvec *
                              (precision == QBX_MIXED ? sizeof(float2) : sizeof(double2));
      if (c.d_zbuf) cudaFree(c.d_zbuf);
      c.d_zbuf = nullptr;
      QBX_CUDA(cudaMalloc(&c.d_zbuf, per_pair * c.pair_batch));
      c.zbuf_bytes = per_pair * c.pair_batch;
    }
    c.precision = precision;
    drop_graphs(c);
    alloc_mixed(c);
  });
}

int qbx_set_cell(qbx_context* h, const double cell[9], double ecut, int nst, const char* xc) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(cell && ecut > 0.0 && nst > 0, 1, "bad cell, ecut or band count");
    const std::string x = xc ? xc : "LDA";
    QBX_REQUIRE(x == "LDA" || x == "PBE", 1, "xc must be LDA or PBE");
    free_atoms(c);
    free_cell(c);
    c.xc = x;
    build_basis(c.wb, cell, ecut);
    build_basis(c.vb, cell, 4.0 * ecut);
    int np[3];
    dense_grid(cell, ecut, np);
    set_grid(c.wb, np[0], np[1], np[2]);
    set_grid(c.vb, np[0], np[1], np[2]);
    upload_sticks(c.dws, c.wb);
    upload_sticks(c.dvs, c.vb);
    c.nst = nst;
    c.occ.assign(nst, 2.0);
    c.extrapolate = false;
    const int ngw = c.wb.ng, ngv = c.vb.ng;
    const size_t N = c.N();
    c.d_gx_w = dupload(c.wb.gx);
    c.d_g2_w = dupload(c.wb.g2);
    c.d_gx_v = dupload(c.vb.gx);
    c.d_g2i_v = dupload(c.vb.g2i);
    const size_t wf = 2 * (size_t)ngw * nst;
    c.d_c = dalloc<double>(wf);
    c.d_hc = dalloc<double>(wf);
    c.d_c_last = dalloc<double>(wf);
    c.d_dc_last = dalloc<double>(wf);
    c.d_ctmp = dalloc<double>(wf);
    QBX_CUDA(cudaMemset(c.d_c, 0, wf * sizeof(double)));
    c.d_occ = dupload(c.occ);
    c.d_prec = dalloc<double>(nst);
    c.d_rhor = dalloc<double>(N);
    c.d_vr = dalloc<double>(N);
    c.d_vxc = dalloc<double>(N);
    c.d_exc = dalloc<double>(N);
    c.d_vx2 = dalloc<double>(N);
    c.d_grad = dalloc<double>(3 * N);
    QBX_CUDA(cudaMalloc(&c.d_grid, N * sizeof(double2)));
    c.d_rhog = dalloc<double>(2 * (size_t)ngv);
    c.d_vion = nullptr;
    c.d_rhops = dalloc<double>(2 * (size_t)ngv);
    c.d_vtmp_g = dalloc<double>(2 * (size_t)ngv);
    c.d_vtmp_g2 = dalloc<double>(2 * (size_t)ngv);
    c.d_xc_g = dalloc<double>(6 * (size_t)ngv);
    const size_t nn = (size_t)nst * nst;
    c.d_nn = dalloc<double>(nn);
    c.d_nn2 = dalloc<double>(nn);
    c.d_nn3 = dalloc<double>(nn);
    c.d_nn4 = dalloc<double>(3 * nn);
    c.d_nn5 = dalloc<double>(nn);
    c.d_ipiv = dalloc<int>(nst);
    c.d_info = dalloc<int>(1);
    int lw1 = 0, lw2 = 0;
    QBX_SOLVER(cusolverDnDpotrf_bufferSize(c.solver, CUBLAS_FILL_MODE_LOWER, nst, c.d_nn, nst, &lw1));
    QBX_SOLVER(cusolverDnDgetrf_bufferSize(c.solver, nst, nst, c.d_nn, nst, &lw2));
    c.solver_lwork = std::max(lw1, lw2);
    c.d_solver_work = dalloc<double>(std::max(1, c.solver_lwork));
    c.d_red = dalloc<double>(4 * 1024);
    c.d_scalars = dalloc<double>(kSlots + nst);
    QBX_CUDA(cudaMemset(c.d_scalars, 0, kSlots * sizeof(double)));
    upload_weights(c);
    // staged FFT stick buffer: bounded to ~4 GB per batch of band pairs
    const int npairs = (nst + 1) / 2;
    const size_t per_pair = (size_t)c.wb.n2 * c.wb.nvec *
                            (c.precision == QBX_MIXED ? sizeof(float2) : sizeof(double2));
    c.pair_batch = (int)std::max<size_t>(1, std::min<size_t>(npairs, ((size_t)4 << 30) / per_pair));
    QBX_CUDA(cudaMalloc(&c.d_zbuf, per_pair * c.pair_batch));
    c.zbuf_bytes = per_pair * c.pair_batch;
    // the specialised FFTs work through a smaller stick buffer that can stay
    // in L2 between the z and plane kernels (64 MB unless overridden)
    {
      size_t mb = 256;
      if (const char* e = std::getenv("QBX_FAST_ZBUF_MB")) mb = std::max(1, std::atoi(e));
      const size_t pp64 = (size_t)c.wb.n2 * c.wb.nvec * sizeof(double2);
      c.zfast_bytes = std::max(mb << 20, pp64);
      QBX_CUDA(cudaMalloc(&c.d_zfast, c.zfast_bytes));
      c.d_vr32 = dalloc<float>(N);
      c.fast_fft = true;
      if (const char* e = std::getenv("QBX_FAST_FFT")) c.fast_fft = std::atoi(e) != 0;
      if (const char* e = std::getenv("QBX_FAST_WARPS")) c.fast_warps = std::max(1, std::min(16, std::atoi(e)));
      if (const char* e = std::getenv("QBX_FAST_RODS")) c.fast_rods = std::max(1, std::min(32, std::atoi(e)));
      if (const char* e = std::getenv("QBX_FAST_CHUNKS")) c.fast_chunks = std::max(1, std::atoi(e));
      c.fast_batch = 16;
      if (const char* e = std::getenv("QBX_FAST_BATCH")) c.fast_batch = std::max(0, std::atoi(e));
      if (const char* e = std::getenv("QBX_FAST_LANE_SHAPE"))
        c.fast_lane_shape = std::max(-1, std::min(6, std::atoi(e)));
      if (const char* e = std::getenv("QBX_FAST_DENSITY_LANE_SHAPE"))
        c.fast_density_lane_shape = (std::atoi(e) == 3 || std::atoi(e) >= 5) && std::atoi(e) <= 8
                                        ? std::atoi(e) : 2;
      if (const char* e = std::getenv("QBX_PSIR")) c.psir_mode = std::atoi(e) != 0 ? 1 : 0;
      if (const char* e = std::getenv("QBX_FWD_STAGED")) c.fast_fwd_staged = std::atoi(e) != 0 ? 1 : 0;
      if (const char* e = std::getenv("QBX_FFT_PRUNE")) c.fast_prune = std::atoi(e) != 0 ? 1 : 0;
      if (const char* e = std::getenv("QBX_ZLANE")) c.fast_zlane = std::max(0, std::min(3, std::atoi(e)));
      if (const char* e = std::getenv("QBX_FWD_PAIRS_PER_CTA"))
        c.fast_fwd_ppc = std::max(1, std::min(64, std::atoi(e)));
      if (const char* e = std::getenv("QBX_FAST_VPSI_SHAPE"))
        c.fast_vpsi_shape = std::max(0, std::min(2, std::atoi(e)));
    }
    c.species.clear();
    c.tau.clear();
    QBX_CUDA(cudaDeviceSynchronize());   // memsets above ran on the legacy stream
    c.have_cell = true;
    alloc_mixed(c);
  });
}

int qbx_basis_sizes(const qbx_context* h, int* ngw, int* ngv, int np[3]) {
  if (!h || !h->c.have_cell) return 7;
  if (ngw) *ngw = h->c.wb.ng;
  if (ngv) *ngv = h->c.vb.ng;
  if (np) { np[0] = h->c.wb.n0; np[1] = h->c.wb.n1; np[2] = h->c.wb.n2; }
  return 0;
}

int qbx_basis_miller(const qbx_context* h, int* hkl) {
  if (!h || !h->c.have_cell || !hkl) return 7;
  std::memcpy(hkl, h->c.wb.hkl.data(), sizeof(int) * h->c.wb.hkl.size());
  return 0;
}

int qbx_set_coeff_order(qbx_context* h, const int* hkl) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    dfree(h->d_perm);
    h->perm.clear();
    if (!hkl) return;
    const int ngw = c.wb.ng;
    std::map<std::tuple<int, int, int>, int> pos;
    for (int i = 0; i < ngw; i++)
      pos[std::make_tuple(c.wb.hkl[3 * i], c.wb.hkl[3 * i + 1], c.wb.hkl[3 * i + 2])] = i;
    h->perm.resize(ngw);
    std::vector<char> seen(ngw, 0);
    for (int i = 0; i < ngw; i++) {
      auto it = pos.find(std::make_tuple(hkl[3 * i], hkl[3 * i + 1], hkl[3 * i + 2]));
      QBX_REQUIRE(it != pos.end(), 14, "Miller index not in the basis");
      QBX_REQUIRE(!seen[it->second], 14, "repeated Miller index");
      seen[it->second] = 1;
      h->perm[i] = it->second;
    }
    h->d_perm = dupload(h->perm);
  });
}

int qbx_add_species(qbx_context* h, int zval, double mesh_spacing, int nmesh, const double* vlocal,
                    int nproj, const int* proj_l, const double* proj, const double* dmat,
                    int* isp) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(zval > 0 && vlocal && nmesh > 8, 1, "bad species data");
    QBX_REQUIRE(nproj == 0 || (proj_l && proj), 1, "missing projector data");
    SpeciesTables s;
    species_from_radial(s, zval, mesh_spacing, nmesh, vlocal, nproj, proj_l, proj, dmat);
    c.species.push_back(s);
    if (isp) *isp = (int)c.species.size() - 1;
  });
}

int qbx_set_atoms(qbx_context* h, const int* na, const double* tau) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(!c.species.empty(), 7, "no species defined");
    const int nsp = (int)c.species.size();
    free_atoms(c);
    c.tau.assign(nsp, std::vector<double>());
    int off = 0, nel = 0, natoms = 0;
    for (int is = 0; is < nsp; is++) {
      QBX_REQUIRE(na[is] >= 0, 1, "negative atom count");
      c.tau[is].assign(tau + 3 * off, tau + 3 * (off + na[is]));
      off += na[is];
      nel += (int)c.species[is].zval * na[is];
    }
    natoms = off;
    (void)nel;   // a net charge is allowed, as in the reference
    // projector columns: species, then projector (l,m), then atom
    c.nproj = 0;
    c.proj_dfac.clear();
    std::vector<int> patom, pcol;
    int atom0 = 0, nrad = 0;
    for (int is = 0; is < nsp; is++) {
      const SpeciesTables& sp = c.species[is];
      for (size_t iop = 0; iop < sp.proj_l.size(); iop++) {
        for (int m = 0; m < 2 * sp.proj_l[iop] + 1; m++)
          for (int ia = 0; ia < na[is]; ia++) {
            c.proj_dfac.push_back(sp.proj_d[iop]);
            patom.push_back(atom0 + ia);
            pcol.insert(pcol.end(), {sp.proj_l[iop], m, nrad, atom0 + ia});
            c.nproj++;
          }
        nrad++;
      }
      atom0 += na[is];
    }
    const int ngw = c.wb.ng, ngv = c.vb.ng;
    if (c.nproj) {
      c.d_anl = dalloc<double>(2 * (size_t)ngw * c.nproj);
      c.d_fnl = dalloc<double>((size_t)c.nproj * c.nst);
      c.d_dfnl = dalloc<double>((size_t)c.nproj * c.nst);
      c.d_pdfac = dupload(c.proj_dfac);
      c.d_patom = dupload(patom);
      c.d_pcol = dupload(pcol);
      // radial projector tables V_nl(|G|), dV_nl/dG on the wavefunction
      // sphere (Species::dvnlg, src/Species.cpp:1172-1185) for the stress
      std::vector<double> vnl((size_t)nrad * ngw), dvnl((size_t)nrad * ngw);
      int r = 0;
      for (int is = 0; is < nsp; is++)
        for (size_t iop = 0; iop < c.species[is].proj_l.size(); iop++, r++)
          for (int ig = 0; ig < ngw; ig++)
            c.species[is].dvnlg((int)iop, c.wb.g[ig], vnl[(size_t)r * ngw + ig],
                                dvnl[(size_t)r * ngw + ig]);
      c.d_vnl = dupload(vnl);
      c.d_dvnl = dupload(dvnl);
    }
    {
      std::vector<double> tall;
      for (int is = 0; is < nsp; is++) tall.insert(tall.end(), c.tau[is].begin(), c.tau[is].end());
      c.d_tau_all = dupload(tall);
      // phase tables of all atoms: 3 axes of 2 hmax + 1 Miller indices each
      const int hmax = std::max(c.vb.n0, std::max(c.vb.n1, c.vb.n2)) / 2 + 1;
      c.phase_tab_bytes = (size_t)std::max(1, natoms) * 3 * (2 * (size_t)hmax + 1) * 16;
      c.d_phase_tab = dalloc<double>(c.phase_tab_bytes / sizeof(double));
      c.fpart_elems = 3 * (size_t)std::max(1, natoms) * 16;
      c.d_fpart = dalloc<double>(c.fpart_elems);
    }
    c.d_fion = dalloc<double>(3 * std::max(1, natoms));
    QBX_CUDA(cudaMallocHost(&c.h_fion, 3 * std::max(1, natoms) * sizeof(double)));
    // species tables on the density sphere (EnergyFunctional::cell_moved,
    // src/EnergyFunctional.cpp:1200-1245)
    std::vector<double> vps((size_t)ngv * nsp), rhops((size_t)ngv * nsp), dvps((size_t)ngv * nsp);
    for (int is = 0; is < nsp; is++)
      for (int ig = 0; ig < ngv; ig++) {
        double v, dv;
        c.species[is].dvlocg(c.vb.g[ig], v, dv);
        vps[(size_t)is * ngv + ig] = v / c.vb.omega;
        dvps[(size_t)is * ngv + ig] = dv / c.vb.omega;
        rhops[(size_t)is * ngv + ig] = c.species[is].rhopsg(c.vb.g[ig]) / c.vb.omega;
      }
    c.d_vps = dupload(vps);
    c.d_dvps = dupload(dvps);
    c.d_rhops_sp = dupload(rhops);
    c.d_sfac = dalloc<double>(2 * (size_t)ngv * nsp);
    if (!c.d_vion) c.d_vion = dalloc<double>(2 * (size_t)ngv);
    launch_setup_atoms(c);
    std::vector<double> zv(nsp);
    c.eself = 0.0;
    for (int is = 0; is < nsp; is++) {
      zv[is] = c.species[is].zval;
      c.eself += na[is] * c.species[is].eself();
    }
    c.esr = esr_energy_forces(c.wb.cell, c.tau, zv, 1.5, c.fion_esr, c.sigma_esr);
    alloc_mixed(c);
    QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

static int set_coeffs_impl(qbx_context* h, const double* src, bool sync, bool reset) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
    if (h->d_perm) {
      QBX_CUDA(cudaMemcpyAsync(c.d_ctmp, src, wf * sizeof(double), cudaMemcpyHostToDevice, c.stream));
      k_permute<<<1184, 256, 0, c.stream>>>((const double2*)c.d_ctmp, h->d_perm, c.wb.ng, c.nst, 1,
                                            (double2*)c.d_c);
      QBX_LAUNCHED(c);
    } else {
      QBX_CUDA(cudaMemcpyAsync(c.d_c, src, wf * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    }
    if (reset) c.extrapolate = false;
    if (sync) QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

static int get_coeffs_impl(qbx_context* h, const double* dsrc, double* dst, bool sync) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
    if (h->d_perm) {
      k_permute<<<1184, 256, 0, c.stream>>>((const double2*)dsrc, h->d_perm, c.wb.ng, c.nst, 0,
                                            (double2*)c.d_ctmp);
      QBX_LAUNCHED(c);
      QBX_CUDA(cudaMemcpyAsync(dst, c.d_ctmp, wf * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    } else {
      QBX_CUDA(cudaMemcpyAsync(dst, dsrc, wf * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    }
    if (sync) QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int qbx_set_coeffs(qbx_context* h, const double* c) { return set_coeffs_impl(h, c, true, true); }
int qbx_set_coeffs_async(qbx_context* h, const double* c) { return set_coeffs_impl(h, c, false, false); }
int qbx_get_coeffs(qbx_context* h, double* c) {
  return h ? get_coeffs_impl(h, h->c.d_c, c, true) : 1;
}
int qbx_get_coeffs_async(qbx_context* h, double* c) {
  return h ? get_coeffs_impl(h, h->c.d_c, c, false) : 1;
}
int qbx_get_hpsi(qbx_context* h, double* hc) {
  return h ? get_coeffs_impl(h, h->c.d_hc, hc, true) : 1;
}

// ---- streamed SlaterDet: copies on their own streams, ordered by events
static void ensure_streaming(Context& c) {
  if (!c.s_in) {
    QBX_CUDA(cudaStreamCreateWithFlags(&c.s_in, cudaStreamNonBlocking));
    QBX_CUDA(cudaStreamCreateWithFlags(&c.s_out, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&c.ev_in, &c.ev_cin_free, &c.ev_step, &c.ev_out})
      QBX_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  if (!c.d_cin) {
    const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
    c.d_cin = dalloc<double>(wf);
    c.d_cout = dalloc<double>(wf);
  }
}

int qbx_stream_in(qbx_context* h, const double* src) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(src && c.kpts.empty(), 1, "streamed coefficients need a host buffer at Gamma");
    ensure_streaming(c);
    // the previous step has taken its input out of the staging buffer
    QBX_CUDA(cudaStreamWaitEvent(c.s_in, c.ev_cin_free, 0));
    QBX_CUDA(cudaMemcpyAsync(c.d_cin, src, 2 * (size_t)c.wb.ng * c.nst * sizeof(double),
                             cudaMemcpyHostToDevice, c.s_in));
    QBX_CUDA(cudaEventRecord(c.ev_in, c.s_in));
    c.in_pending = true;
  });
}

int qbx_scf_step_async(qbx_context* h) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(c.kpts.empty(), 1, "the streamed step is not available at k points off Gamma");
    ensure_streaming(c);
    const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
    if (c.in_pending) {
      QBX_CUDA(cudaStreamWaitEvent(c.stream, c.ev_in, 0));
      if (h->d_perm) {
        k_permute<<<1184, 256, 0, c.stream>>>((const double2*)c.d_cin, h->d_perm, c.wb.ng, c.nst,
                                              1, (double2*)c.d_c);
        QBX_LAUNCHED(c);
      } else {
        QBX_CUDA(cudaMemcpyAsync(c.d_c, c.d_cin, wf * sizeof(double), cudaMemcpyDeviceToDevice,
                                 c.stream));
      }
      QBX_CUDA(cudaEventRecord(c.ev_cin_free, c.stream));
      c.in_pending = false;
    }
    StepGraph& g = c.graphs[c.extrapolate ? 1 : 0];
    if (c.step_graph && c.wf_dyn == 0 && !c.prof.on && g.exec) {
      // captured: launch and return; the host finish (energies, status) of
      // this step waits for qbx_stream_wait or the next uncaptured step
      launch_step_graph(c, g);
      c.extrapolate = true;         // as finish_graph_step leaves it
      c.finish_pending = true;
    } else {
      // not captured (yet): the synchronous step, which may capture
      QBX_CUDA(cudaStreamSynchronize(c.stream));
      if (c.finish_pending) finish_graph_step(c, false, c.last_energies, nullptr);
      c.finish_pending = false;
      scf_step_any(c, false, false, c.last_energies, nullptr);
    }
    // the result to its staging buffer once the previous download is done
    QBX_CUDA(cudaStreamWaitEvent(c.stream, c.ev_out, 0));
    if (h->d_perm) {
      k_permute<<<1184, 256, 0, c.stream>>>((const double2*)c.d_c, h->d_perm, c.wb.ng, c.nst, 0,
                                            (double2*)c.d_cout);
      QBX_LAUNCHED(c);
    } else {
      QBX_CUDA(cudaMemcpyAsync(c.d_cout, c.d_c, wf * sizeof(double), cudaMemcpyDeviceToDevice,
                               c.stream));
    }
    QBX_CUDA(cudaEventRecord(c.ev_step, c.stream));
  });
}

int qbx_stream_out(qbx_context* h, double* dst) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(dst && c.s_out, 1, "qbx_stream_out before a streamed step");
    QBX_CUDA(cudaStreamWaitEvent(c.s_out, c.ev_step, 0));
    QBX_CUDA(cudaMemcpyAsync(dst, c.d_cout, 2 * (size_t)c.wb.ng * c.nst * sizeof(double),
                             cudaMemcpyDeviceToHost, c.s_out));
    QBX_CUDA(cudaEventRecord(c.ev_out, c.s_out));
  });
}

int qbx_stream_wait(qbx_context* h, double* energies) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    if (c.s_in) QBX_CUDA(cudaStreamSynchronize(c.s_in));
    if (c.s_out) QBX_CUDA(cudaStreamSynchronize(c.s_out));
    if (c.finish_pending) {
      finish_graph_step(c, false, c.last_energies, nullptr);
      c.finish_pending = false;
    }
    QBX_REQUIRE(std::isfinite(c.last_energies[8]), 41, "streamed step: total energy not finite");
    if (energies) std::memcpy(energies, c.last_energies, sizeof(double) * QBX_NENERGY);
  });
}

int qbx_set_kpoints(qbx_context* h, int nkp, const double* kpoints, const double* weights) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(nkp >= 0 && (nkp == 0 || (kpoints && weights)), 1, "bad k point arguments");
    drop_graphs(c);
    set_kpoints(c, nkp, kpoints, weights);
  });
}

static KPointSet& kpoint_of(Context& c, int ikp) {
  QBX_REQUIRE(ikp >= 0 && ikp < (int)c.kpts.size(), 1, "no such k point");
  return c.kpts[ikp];
}

int qbx_kpoint_basis(const qbx_context* h, int ikp, int* ngw, int* hkl) {
  return guarded(const_cast<qbx_context*>(h), [&](Context& c) {
    const KPointSet& kp = kpoint_of(c, ikp);
    if (ngw) *ngw = kp.kb.ng;
    if (hkl) std::memcpy(hkl, kp.kb.hkl.data(), sizeof(int) * kp.kb.hkl.size());
  });
}

int qbx_set_kpoint_coeffs(qbx_context* h, int ikp, const double* src) {
  return guarded(h, [&](Context& c) {
    KPointSet& kp = kpoint_of(c, ikp);
    QBX_REQUIRE(src, 1, "null coefficients");
    const size_t n = 2 * (size_t)kp.kb.ng * c.nst;
    QBX_CUDA(cudaMemcpyAsync(kp.d_c, src, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    c.kpts_extrapolate = false;   // a new wavefunction starts a new history
  });
}

static int get_kpoint_impl(qbx_context* h, int ikp, bool hpsi, double* dst) {
  return guarded(h, [&](Context& c) {
    KPointSet& kp = kpoint_of(c, ikp);
    QBX_REQUIRE(dst, 1, "null output");
    const size_t n = 2 * (size_t)kp.kb.ng * c.nst;
    QBX_CUDA(cudaMemcpyAsync(dst, hpsi ? kp.d_hc : kp.d_c, n * sizeof(double),
                             cudaMemcpyDeviceToHost, c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}
int qbx_get_kpoint_coeffs(qbx_context* h, int ikp, double* c) { return get_kpoint_impl(h, ikp, false, c); }
int qbx_get_kpoint_hpsi(qbx_context* h, int ikp, double* hc) { return get_kpoint_impl(h, ikp, true, hc); }

int qbx_gram(qbx_context* h) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    if (!c.kpts.empty()) gram_k(c);
    else gram(c);
    readback(c, false);
    check_status(c);
  });
}

int qbx_update_density(qbx_context* h, double* total_charge) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    if (!c.kpts.empty()) update_density_k(c);
    else update_density(c);
    readback(c, false);
    finish_density(c);
    if (total_charge) *total_charge = c.total_charge;
  });
}

int qbx_get_density(qbx_context* h, double* rhor) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_CUDA(cudaMemcpyAsync(rhor, c.d_rhor, c.N() * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int qbx_update_vhxc(qbx_context* h) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    update_vhxc(c);
    readback(c, false);
    finish_vhxc(c);
  });
}

int qbx_get_vr(qbx_context* h, double* vr) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_CUDA(cudaMemcpyAsync(vr, c.d_vr, c.N() * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int qbx_energy(qbx_context* h, int hpsi, int forces, double* energies, double* fion) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    if (!c.kpts.empty()) {
      QBX_REQUIRE(!forces, 1, "forces are not available at k points off Gamma");
      energy_k(c, hpsi != 0);
    } else {
      energy(c, hpsi != 0, forces != 0);
    }
    readback(c, forces != 0);
    check_status(c);
    finish_energy(c, forces != 0);
    fill_energies(c, energies);
    if (forces && fion) std::memcpy(fion, c.fion.data(), sizeof(double) * c.fion.size());
  });
}

int qbx_eigenvalue_sum(qbx_context* h, double* eig) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    if (!c.kpts.empty()) eigsum_k(c);
    else launch_eigsum(c);
    readback(c, false);
    finish_eigsum(c);
    if (eig) *eig = c.eigsum;
  });
}

int qbx_psda_update(qbx_context* h) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    if (!c.kpts.empty()) psda_update_k(c);
    else psda_update(c);
    readback(c, false);
    check_status(c);
    finish_theta(c);
  });
}

int qbx_psda_reset(qbx_context* h) {
  return guarded(h, [&](Context& c) {
    c.extrapolate = false;
    c.kpts_extrapolate = false;
  });
}


}  // extern "C"

namespace qbx {
void scf_step_any(Context& c, bool want_f, bool want_s, double* energies, double* fion) {
  if (StepGraph* g = step_graph_for(c, want_f, want_s)) {
    launch_step_graph(c, *g);
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    finish_graph_step(c, want_f, energies, fion);
    return;
  }
  step_eager(c, want_f, want_s, energies, fion);
}
}  // namespace qbx

extern "C" {
int qbx_scf_step(qbx_context* h, int forces, double* energies, double* fion) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    scf_step_any(c, (forces & 1) != 0, (forces & 2) != 0, energies, fion);
  });
}

int qbx_scf_run(qbx_context* h, int nitscf, int nite, double mix_coeff, double mix_rcut,
                int mix_ndim, double scf_tol, double* etotal_int, double* eigsum,
                int* nite_done, int* nitscf_done) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(c.kpts.empty(), 1, "the charge-mixing SCF loop is not available at k points off Gamma");
    QBX_REQUIRE(nitscf > 0 && nite >= 0 && mix_coeff >= 0.0 && mix_rcut >= 0.0, 1,
                "bad SCF arguments");
    scf_run(c, nitscf, nite, mix_coeff, mix_rcut, mix_ndim, scf_tol, etotal_int, eigsum,
            nite_done, nitscf_done);
  });
}

int qbx_write_wavefunction(qbx_context* h, const char* path) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "the sample wavefunction writer is not available at k points off Gamma");
    QBX_REQUIRE(path, 1, "null path");
    std::ofstream os(path);
    QBX_REQUIRE(os.good(), 75, std::string("cannot write ") + path);
    write_wavefunction(c, os);
    QBX_REQUIRE(os.good(), 75, std::string("write failed: ") + path);
  });
}

int qbx_read_wavefunction(qbx_context* h, const char* path) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "the sample wavefunction reader is not available at k points off Gamma");
    QBX_REQUIRE(path, 1, "null path");
    std::ifstream is(path, std::ios::binary);
    QBX_REQUIRE(is.good(), 75, std::string("cannot read ") + path);
    std::ostringstream ss;
    ss << is.rdbuf();
    read_wavefunction(c, ss.str());
  });
}

int qbx_move_atoms(qbx_context* h, const double* tau) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(tau, 1, "null positions");
    move_atoms(c, tau);
  });
}

int qbx_md_run(qbx_context* h, int niter, int nitscf, double dt, const double* mass_amu,
               double* vel, double* tau_out, double* ionic, double* scf) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(c.kpts.empty(), 1, "molecular dynamics is not available at k points off Gamma");
    QBX_REQUIRE(niter > 0 && nitscf >= 0 && dt != 0.0 && mass_amu, 1, "bad MD arguments");
    for (size_t is = 0; is < c.species.size(); is++)
      QBX_REQUIRE(mass_amu[is] > 0.0, 1, "species mass must be positive");
    md_run(c, niter, nitscf, dt, mass_amu, vel, tau_out, ionic, scf);
  });
}

int qbx_polar(qbx_context* h, double* x, double tol, int maxiter, int graph, int* iters) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(x && maxiter > 0, 1, "bad polar arguments");
    const size_t nn = (size_t)c.nst * c.nst;
    double* d = c.d_nn2;
    QBX_CUDA(cudaMemcpyAsync(d, x, nn * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    const int it = polar_entry(c, d, tol, maxiter, graph != 0);
    QBX_CUDA(cudaMemcpyAsync(x, d, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    readback(c, false);
    check_status(c);
    if (iters) *iters = it;
  });
}

int qbx_lower_inverse(qbx_context* h, int n, const double* l, double* li, int* blocked) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(n > 0 && l && li, 1, "bad triangular-inverse arguments");
    const size_t nn = (size_t)n * n;
    double *dl = dalloc<double>(nn), *dli = dalloc<double>(nn), *dw = dalloc<double>(nn / 4 + 1);
    try {
      QBX_CUDA(cudaMemcpyAsync(dl, l, nn * sizeof(double), cudaMemcpyHostToDevice, c.stream));
      lower_inverse(c, dl, n, dli, dw);
      QBX_CUDA(cudaMemcpyAsync(li, dli, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
      QBX_CUDA(cudaStreamSynchronize(c.stream));
    } catch (...) {
      dfree(dl); dfree(dli); dfree(dw);
      throw;
    }
    dfree(dl); dfree(dli); dfree(dw);
    if (blocked) *blocked = lower_inverse_blocked(n) ? 1 : 0;
  });
}

int qbx_set_step_graph(qbx_context* h, int on) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(!on || !c.shard_comm, 1, "captured steps and band sharding are exclusive");
    c.step_graph = on != 0;
    c.graph_note.clear();
    drop_graphs(c);
  });
}

int qbx_step_graph_info(qbx_context* h, int* captured, long* launches, long* batch_launches,
                        char* note, int note_len) {
  return guarded(h, [&](Context& c) {
    int n = 0;
    for (auto& g : c.graphs) n += g.exec != nullptr;
    if (captured) *captured = n;
    if (launches) *launches = c.graph_launches;
    if (batch_launches) *batch_launches = c.batch_launches;
    if (note && note_len > 0) {
      std::strncpy(note, c.graph_note.c_str(), (size_t)note_len - 1);
      note[note_len - 1] = 0;
    }
  });
}

int qbx_scf_step_batch(qbx_context** ctxs, int n, int compute_forces, double* energies) {
  if (!ctxs || n <= 0) return 1;
  for (int i = 0; i < n; i++)
    if (!ctxs[i]) return 1;
  // When every context has its step captured, one thread launches all the
  // graphs (each on its context's stream, so the GPU runs the systems side
  // by side), then waits for each and forms its energies.
  {
    const bool want_f = (compute_forces & 1) != 0;
    std::vector<StepGraph*> gs(n, nullptr);
    bool all = (compute_forces & 2) == 0;
    for (int i = 0; i < n && all; i++) {
      Context& c = ctxs[i]->c;
      if (!c.step_graph || c.wf_dyn != 0 || c.prof.on || !c.have_cell || c.tau.empty()) {
        all = false;
        break;
      }
      gs[i] = &c.graphs[(c.extrapolate ? 1 : 0) + (want_f ? 2 : 0)];
      all = gs[i]->exec != nullptr;
    }
    if (all) {
      // with QBX_BATCH_GRAPH on the first context: one graph over all
      // members (parallel branches), cached there while the members'
      // captures stay the same
      Context& lead = ctxs[0]->c;
      std::vector<long> ids(n);
      for (int i = 0; i < n; i++) ids[i] = gs[i]->id;
      if (lead.batch_single_graph && lead.batch.ids != ids) {
        // one multi-stream capture: every member's stream joins the lead
        // stream's capture through an event, records its step as a branch
        // and joins back
        drop_batch(lead);
        lead.batch.ids = ids;
        std::string why;
        cudaGraph_t graph = nullptr;
        std::vector<cudaEvent_t> ev(n + 1, nullptr);
        try {
          for (auto& e : ev) QBX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
          QBX_CUDA(cudaSetDevice(lead.device));
          QBX_CUDA(cudaStreamBeginCapture(lead.stream, cudaStreamCaptureModeRelaxed));
          try {
            QBX_CUDA(cudaEventRecord(ev[0], lead.stream));
            for (int i = 0; i < n; i++) {
              Context& c = ctxs[i]->c;
              QBX_REQUIRE(c.device == lead.device, 1, "batch members on different devices");
              if (i > 0) QBX_CUDA(cudaStreamWaitEvent(c.stream, ev[0], 0));
              record_step(c, want_f);
              if (i > 0) {
                QBX_CUDA(cudaEventRecord(ev[i + 1], c.stream));
                QBX_CUDA(cudaStreamWaitEvent(lead.stream, ev[i + 1], 0));
              }
            }
          } catch (...) {
            cudaStreamEndCapture(lead.stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            graph = nullptr;
            throw;
          }
          QBX_CUDA(cudaStreamEndCapture(lead.stream, &graph));
          QBX_CUDA(cudaGraphInstantiate(&lead.batch.exec, graph, 0));
        } catch (const Error& e) {
          why = e.msg;
        }
        if (graph) cudaGraphDestroy(graph);
        for (auto e : ev)
          if (e) cudaEventDestroy(e);
        if (!why.empty()) {
          cudaGetLastError();
          if (lead.batch.exec) cudaGraphExecDestroy(lead.batch.exec);
          lead.batch.exec = nullptr;
          lead.batch.failed = true;
          lead.graph_note = "batch graph: " + why + "; members launched one by one";
        }
      }
      if (lead.batch.exec) {
        const int rc = guarded(ctxs[0], [&](Context& c) {
          QBX_CUDA(cudaGraphLaunch(c.batch.exec, c.stream));
          QBX_CUDA(cudaStreamSynchronize(c.stream));
        });
        if (rc) return rc;
        int first = 0;
        for (int i = 0; i < n; i++) {
          const int r = guarded(ctxs[i], [&](Context& c) {
            c.nlaunch += gs[i]->nkernels;
            c.graph_launches++;
            finish_graph_step(c, want_f,
                              energies ? energies + (size_t)i * QBX_NENERGY : nullptr, nullptr);
          });
          if (r && !first) first = r;
        }
        lead.batch_launches++;
        return first;
      }
      for (int i = 0; i < n; i++) {
        const int rc = guarded(ctxs[i], [&](Context& c) { launch_step_graph(c, *gs[i]); });
        if (rc) return rc;
      }
      int first = 0;
      for (int i = 0; i < n; i++) {
        const int rc = guarded(ctxs[i], [&](Context& c) {
          QBX_CUDA(cudaStreamSynchronize(c.stream));
          finish_graph_step(c, want_f,
                            energies ? energies + (size_t)i * QBX_NENERGY : nullptr, nullptr);
        });
        if (rc && !first) first = rc;
      }
      return first;
    }
  }
  // Otherwise one host thread per context: each drives its own stream, so
  // the GPU overlaps the systems' kernels; the host synchronisations of an
  // eager step stall only their own system.
  std::vector<int> rc(n, 0);
  std::vector<std::thread> th;
  th.reserve(n);
  for (int i = 0; i < n; i++)
    th.emplace_back([&, i]() {
      rc[i] = qbx_scf_step(ctxs[i], compute_forces,
                           energies ? energies + (size_t)i * QBX_NENERGY : nullptr, nullptr);
    });
  for (auto& t : th) t.join();
  for (int i = 0; i < n; i++)
    if (rc[i]) return rc[i];
  return 0;
}

int qbx_set_wf_dyn(qbx_context* h, const char* name) {
  return guarded(h, [&](Context& c) {
    const std::string s = name ? name : "";
    QBX_REQUIRE(s == "PSDA" || s == "JD", 1, "wf_dyn must be PSDA or JD");
    c.wf_dyn = (s == "JD") ? 1 : 0;
    c.extrapolate = false;
    drop_graphs(c);
  });
}

int qbx_jd_update(qbx_context* h) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(c.kpts.empty(), 1, "the JD stepper is not available at k points off Gamma");
    jd_update(c);
    readback(c, false);
    check_status(c);
  });
}

int qbx_autotune(qbx_context* h, char* report, int report_len) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    std::vector<std::pair<std::string, double>> log;
    drop_graphs(c);   // the launch shapes may change
    autotune_fft(c, &log);
    if (report && report_len > 0) {
      std::string r;
      for (auto& e : log) r += e.first + ": " + std::to_string(e.second) + " ms\n";
      r += "chosen: lane " + std::to_string(c.fast_lane_shape) + ", warp " +
           std::to_string(c.fast_vpsi_shape) + ", density lane " +
           std::to_string(c.fast_density_lane_shape) + " x " + std::to_string(c.fast_chunks) +
           ", pairs " +
           std::to_string(c.fast_batch) + ", rods " + std::to_string(c.fast_rods) +
           ", z lanes " + std::to_string(c.fast_zlane) + ", pruned xy " +
           std::to_string(c.fast_prune && c.dws.xw <= prune_width(c.dws.n0) &&
                          c.dws.yw <= prune_width(c.dws.n1)) +
           " z " + std::to_string(c.fast_prune && c.dws.zw <= prune_width(c.dws.n2)) + "\n";
      std::strncpy(report, r.c_str(), (size_t)report_len - 1);
      report[report_len - 1] = 0;
    }
  });
}

static void copy_stress(const Context& c, double* sigma, double* parts) {
  if (sigma) std::memcpy(sigma, c.sigma, sizeof(c.sigma));
  if (parts) std::memcpy(parts, c.sigma_parts, sizeof(c.sigma_parts));
}

int qbx_stress(qbx_context* h, double* sigma, double* parts) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(c.kpts.empty(), 1, "the stress tensor is not available at k points off Gamma");
    compute_stress(c);
    readback(c, false);
    check_status(c);
    finish_stress(c);
    copy_stress(c, sigma, parts);
  });
}

int qbx_get_stress(qbx_context* h, double* sigma, double* parts) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(c.have_stress, 7, "no stress computed yet");
    copy_stress(c, sigma, parts);
  });
}

int qbx_ft_backward_pair(qbx_context* h, int n1, int n2, double* f) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(n1 >= 0 && n1 < c.nst && n2 < c.nst, 1, "band index out of range");
    const size_t N = c.N();
    const double* c1 = c.d_c + 2 * (size_t)n1 * c.wb.ng;
    const double* c2 = n2 >= 0 ? c.d_c + 2 * (size_t)n2 * c.wb.ng : nullptr;
    wb_backward_pair(c, c1, c2, c.d_grad);   // complex grid in the first 2N of d_grad
    QBX_CUDA(cudaMemcpyAsync(f, c.d_grad, 2 * N * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

// ---------------------------------------------- class-level entry points
// SlaterDet and NonLocalPotential operations on the caller's host arrays
// (coefficients in the caller's row order when qbx_set_coeff_order was
// given, grids x fastest), for callers that keep the reference's classes.

namespace {

__global__ void k_sub_kinetic(double2* __restrict__ hc, const double2* __restrict__ c,
                              const double* __restrict__ g2, int ng, int nst) {
  const size_t n = (size_t)ng * nst;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const double k = 0.5 * g2[t % ng];
    const double2 a = c[t];
    hc[t].x -= k * a.x;
    hc[t].y -= k * a.y;
  }
}

// d = 2 sum_n sum_i a_n[i] b_n[i] - sum_n a_n[0] b_n[0] over the real view
// (2 ng doubles per band), the G = 0 row at internal index 0
__global__ void k_sd_dot(const double* __restrict__ a, const double* __restrict__ b, int ng,
                         int nst, double* __restrict__ out) {
  __shared__ double sh[32];
  const size_t n = 2 * (size_t)ng * nst;
  double s = 0.0;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t i = t % (2 * (size_t)ng);
    const double p = a[t] * b[t];
    s += i == 0 ? p : 2.0 * p;   // the first real element of each band once
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
    atomicAdd(out, t);
  }
}

double* lazy_wf(Context& c, double*& p) {
  if (!p) p = dalloc<double>(2 * (size_t)c.wb.ng * c.nst);
  return p;
}

// host (caller order) -> device (internal order)
void upload_wf(qbx_context* h, const double* src, double* dst) {
  Context& c = h->c;
  const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
  if (h->d_perm) {
    QBX_CUDA(cudaMemcpyAsync(c.d_ctmp, src, wf * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    k_permute<<<1184, 256, 0, c.stream>>>((const double2*)c.d_ctmp, h->d_perm, c.wb.ng, c.nst, 1,
                                          (double2*)dst);
    QBX_LAUNCHED(c);
  } else {
    QBX_CUDA(cudaMemcpyAsync(dst, src, wf * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  }
}

// device (internal order) -> host vector (caller order)
std::vector<double> download_wf(qbx_context* h, const double* dsrc) {
  Context& c = h->c;
  const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
  std::vector<double> out(wf);
  const double* src = dsrc;
  if (h->d_perm) {
    k_permute<<<1184, 256, 0, c.stream>>>((const double2*)dsrc, h->d_perm, c.wb.ng, c.nst, 0,
                                          (double2*)c.d_ctmp);
    QBX_LAUNCHED(c);
    src = c.d_ctmp;
  }
  QBX_CUDA(cudaMemcpyAsync(out.data(), src, wf * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  QBX_CUDA(cudaStreamSynchronize(c.stream));
  return out;
}

}  // namespace

int qbx_compute_density(qbx_context* h, double weight, double* rho) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "qbx_compute_density works on the Gamma SlaterDet");
    QBX_REQUIRE(rho, 1, "null density array");
    const size_t N = c.N();
    if (!c.d_xgrid) c.d_xgrid = dalloc<double>(N);
    launch_density(c, c.d_c, c.d_xgrid);
    std::vector<double> tmp(N);
    QBX_CUDA(cudaMemcpyAsync(tmp.data(), c.d_xgrid, N * sizeof(double), cudaMemcpyDeviceToHost,
                             c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    for (size_t i = 0; i < N; i++) rho[i] += weight * tmp[i];
  });
}

int qbx_rs_mul_add(qbx_context* h, const double* v, double* dc) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "qbx_rs_mul_add works on the Gamma SlaterDet");
    QBX_REQUIRE(v && dc, 1, "null potential or output array");
    const size_t N = c.N();
    if (!c.d_xgrid) c.d_xgrid = dalloc<double>(N);
    double* out = lazy_wf(c, c.d_xsd);
    QBX_CUDA(cudaMemcpyAsync(c.d_xgrid, v, N * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    launch_vpsi(c, c.d_c, c.d_xgrid, out);   // 1/2 G^2 c + V psi
    k_sub_kinetic<<<1184, 256, 0, c.stream>>>((double2*)out, (const double2*)c.d_c, c.d_g2_w,
                                              c.wb.ng, c.nst);
    QBX_LAUNCHED(c);
    const std::vector<double> add = download_wf(h, out);
    for (size_t i = 0; i < add.size(); i++) dc[i] += add[i];
  });
}

int qbx_nonlocal_energy(qbx_context* h, int compute_hpsi, double* dc, int compute_forces,
                        double* fion, int compute_stress, double* sigma_enl, double* enl) {
  return guarded(h, [&](Context& c) {
    check_ready(c, true);
    QBX_REQUIRE(c.kpts.empty(), 1, "qbx_nonlocal_energy works on the Gamma SlaterDet");
    QBX_REQUIRE(!compute_hpsi || dc, 1, "null H*psi array");
    QBX_REQUIRE(!compute_forces || fion, 1, "null force array");
    QBX_REQUIRE(!compute_stress || sigma_enl, 1, "null stress array");
    double* out = compute_hpsi ? lazy_wf(c, c.d_xsd) : nullptr;
    nonlocal_only(c, compute_hpsi != 0, out);
    size_t natoms = 0;
    for (auto& t : c.tau) natoms += t.size() / 3;
    if (compute_forces) {
      QBX_CUDA(cudaMemsetAsync(c.d_fion, 0, sizeof(double) * 3 * natoms, c.stream));
      if (c.nproj) launch_nl_forces(c, c.d_fion);
    }
    if (compute_stress) compute_stress_nl(c);
    readback(c, compute_forces != 0);
    check_status(c);
    const double e_nl = c.nproj ? c.h_scalars[SLOT_ENL] : 0.0;
    if (enl) *enl = e_nl;
    if (compute_forces) std::memcpy(fion, c.h_fion, sizeof(double) * 3 * natoms);
    if (compute_stress) nl_stress_part(c, e_nl, sigma_enl);
    if (compute_hpsi) {
      const std::vector<double> add = download_wf(h, out);
      for (size_t i = 0; i < add.size(); i++) dc[i] += add[i];
    }
  });
}

int qbx_ortho_align(qbx_context* h, const double* c_ref) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "qbx_ortho_align works on the Gamma SlaterDet");
    QBX_REQUIRE(c_ref, 1, "null coefficient array");
    upload_wf(h, c_ref, c.d_c_last);
    if (c.precision == MIXED)
      split_bf16_2d(c, c.d_c_last, 2 * c.wb.ng, c.nst, 2 * c.wb.ng, c.cs_hi[0], c.cs_lo[0], c.ldp);
    ortho_align(c);
    // the stepper's last-step buffer now holds the caller's SlaterDet
    c.extrapolate = false;
    readback(c, false);
    check_status(c);
  });
}

int qbx_diag(qbx_context* h, int eigvec, double* eig) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "qbx_diag works on the Gamma SlaterDet");
    QBX_REQUIRE(eig, 1, "null eigenvalue array");
    double* w = dalloc<double>(c.nst);
    try {
      diag(c, eigvec != 0, w);
      QBX_CUDA(cudaMemcpy(eig, w, sizeof(double) * c.nst, cudaMemcpyDeviceToHost));
    } catch (...) {
      dfree(w);
      throw;
    }
    dfree(w);
  });
}

int qbx_dot(qbx_context* h, const double* c_other, double* d) {
  return guarded(h, [&](Context& c) {
    check_ready(c, false);
    QBX_REQUIRE(c.kpts.empty(), 1, "qbx_dot works on the Gamma SlaterDet");
    QBX_REQUIRE(c_other && d, 1, "null coefficient or result pointer");
    double* other = lazy_wf(c, c.d_xsd);
    upload_wf(h, c_other, other);
    double* acc = c.d_scalars + SLOT_SCRATCH;
    QBX_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), c.stream));
    k_sd_dot<<<1184, 256, 0, c.stream>>>(c.d_c, other, c.wb.ng, c.nst, acc);
    QBX_LAUNCHED(c);
    QBX_CUDA(cudaMemcpyAsync(d, acc, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int qbx_profile(qbx_context* h, int on) {
  return guarded(h, [&](Context& c) {
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    c.prof.reset();
    c.prof.on = (on != 0);
  });
}

int qbx_profile_get(qbx_context* h, const char* name, double* ms, long* count) {
  return guarded(h, [&](Context& c) {
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    c.prof.resolve();
    double t = 0.0;
    long n = 0;
    for (size_t i = 0; i < c.prof.names.size(); i++)
      if (c.prof.names[i] == name) { t = c.prof.ms[i]; n = c.prof.count[i]; }
    if (ms) *ms = t;
    if (count) *count = n;
  });
}

int qbx_launch_count(qbx_context* h, long* n) {
  if (!h) return 1;
  if (n) *n = h->c.nlaunch;
  return 0;
}

void* qbx_stream(qbx_context* h) { return h ? (void*)h->c.stream : nullptr; }

int qbx_split_gemm_tn(qbx_context* h, int m, int n, int k, const double* a, const double* b,
                      double* d, int backend) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(m > 0 && n > 0 && k > 0 && a && b && d, 1, "bad GEMM arguments");
    QBX_REQUIRE(backend >= 0 && backend <= 4, 1, "backend must be 0 to 4");
    double *da = dalloc<double>((size_t)k * m), *db = dalloc<double>((size_t)k * n);
    double* dd = dalloc<double>((size_t)m * n);
    void *ah = nullptr, *al = nullptr, *bh = nullptr, *bl = nullptr, *acc = nullptr;
    const int saved = c.gemm_backend;
    const size_t saved_acc = c.acc32_elems;
    void* saved_ptr = c.d_acc32;
    auto cleanup = [&]() {
      c.gemm_backend = saved; c.d_acc32 = saved_ptr; c.acc32_elems = saved_acc;
      if (acc) cudaFree(acc);
      if (ah) cudaFree(ah);
      if (al) cudaFree(al);
      if (bh) cudaFree(bh);
      if (bl) cudaFree(bl);
      dfree(da); dfree(db); dfree(dd);
    };
    try {
      h2d_sync(da, a, sizeof(double) * k * m);
      h2d_sync(db, b, sizeof(double) * k * n);
      if (backend == 3 || backend == 4) {
        // A as an MN-major operand (its transposed split, m contiguous), B
        // K-major: the tall-update form, BF16 (3) or TF32 (4) splits
        const int kind = backend == 3 ? TALL_BF16 : TALL_TF32;
        const size_t es = backend == 3 ? 2 : 4;
        const int ldm = (m + 63) / 64 * 64, ldk = (k + 63) / 64 * 64;
        QBX_CUDA(cudaMalloc(&ah, (size_t)ldm * k * es));
        QBX_CUDA(cudaMalloc(&al, (size_t)ldm * k * es));
        QBX_CUDA(cudaMalloc(&bh, (size_t)ldk * n * es));
        QBX_CUDA(cudaMalloc(&bl, (size_t)ldk * n * es));
        split_t(c, kind, da, k, m, k, ah, al, ldm);
        split_plain(c, kind, db, k, n, k, bh, bl, ldk);
        QBX_CUDA(cudaMemsetAsync(dd, 0, sizeof(double) * m * n, c.stream));
        tc_gemm_kind_nn_mn(c, kind, m, n, k, 1.0, ah, al, ldm, bh, bl, ldk, 0.0, dd, m);
      } else if (backend == 2) {
        // TF32 splits through the tcgen05 kind::tf32 kernel
        const int ldk = pad4(k);
        QBX_CUDA(cudaMalloc(&ah, (size_t)ldk * m * 4));
        QBX_CUDA(cudaMalloc(&al, (size_t)ldk * m * 4));
        QBX_CUDA(cudaMalloc(&bh, (size_t)ldk * n * 4));
        QBX_CUDA(cudaMalloc(&bl, (size_t)ldk * n * 4));
        split_tf32(c, da, k, m, k, (float*)ah, (float*)al, ldk);
        split_tf32(c, db, k, n, k, (float*)bh, (float*)bl, ldk);
        QBX_CUDA(cudaMemsetAsync(dd, 0, sizeof(double) * m * n, c.stream));
        tc_tf32_gemm_tn(c, m, n, k, 1.0, (const float*)ah, (const float*)al, ldk,
                        (const float*)bh, (const float*)bl, ldk, 0.0, dd, m);
      } else {
        const int ldp = (k + 63) / 64 * 64;
        QBX_CUDA(cudaMalloc(&ah, (size_t)ldp * m * 2));
        QBX_CUDA(cudaMalloc(&al, (size_t)ldp * m * 2));
        QBX_CUDA(cudaMalloc(&bh, (size_t)ldp * n * 2));
        QBX_CUDA(cudaMalloc(&bl, (size_t)ldp * n * 2));
        split_bf16_2d(c, da, k, m, k, ah, al, ldp);
        split_bf16_2d(c, db, k, n, k, bh, bl, ldp);
        QBX_CUDA(cudaMalloc(&acc, (size_t)m * n * sizeof(float)));
        c.d_acc32 = acc;
        c.acc32_elems = (size_t)m * n;
        c.gemm_backend = backend;
        QBX_REQUIRE(backend == 0 || tc_gemm_supported(c, true, false, m, n, k), 54,
                    "shape not supported by the tcgen05 GEMM");
        split_gemm(c, true, false, m, n, k, 1.0, ah, al, ldp, bh, bl, ldp, 0.0, dd);
      }
      QBX_CUDA(cudaMemcpyAsync(d, dd, sizeof(double) * m * n, cudaMemcpyDeviceToHost, c.stream));
      QBX_CUDA(cudaStreamSynchronize(c.stream));
      QBX_REQUIRE(tc_check_error(c) == 0, 55, "tcgen05 GEMM pipeline wait timed out");
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

int qbx_set_gemm_backend(qbx_context* h, int backend) {
  return guarded(h, [&](Context& c) {
    QBX_REQUIRE(backend == 0 || backend == 1, 1, "backend must be 0 (cuBLAS) or 1 (tcgen05)");
    const bool changed = c.gemm_backend != backend;
    c.gemm_backend = backend;
    drop_graphs(c);
    // the cuBLAS backend has TF32 split buffers of its own
    if (changed && c.have_cell) alloc_mixed(c);
  });
}

int qbx_synchronize(qbx_context* h) {
  return guarded(h, [&](Context& c) { QBX_CUDA(cudaStreamSynchronize(c.stream)); });
}

int qbx_host_basis(const double cell[9], double ecut, int* ngw, int* ngv, int np[3], int* hkl) {
  try {
    Basis w, v;
    build_basis(w, cell, ecut);
    build_basis(v, cell, 4.0 * ecut);
    int g[3];
    dense_grid(cell, ecut, g);
    if (ngw) *ngw = w.ng;
    if (ngv) *ngv = v.ng;
    if (np) { np[0] = g[0]; np[1] = g[1]; np[2] = g[2]; }
    if (hkl) std::memcpy(hkl, w.hkl.data(), sizeof(int) * w.hkl.size());
    return 0;
  } catch (const Error& e) {
    return e.code;
  } catch (...) {
    return 6;
  }
}

int qbx_host_kbasis(const double cell[9], double ecut, const double k[3], int* ngw, int* first,
                    int* hkl) {
  try {
    Basis b;
    build_kbasis(b, cell, ecut, k);
    if (ngw) *ngw = b.ng;
    if (first) *first = b.first;
    if (hkl) std::memcpy(hkl, b.hkl.data(), sizeof(int) * b.hkl.size());
    return 0;
  } catch (const Error& e) {
    return e.code;
  } catch (...) {
    return 6;
  }
}

int qbx_host_species_eval(int zval, double mesh_spacing, int nmesh, const double* vlocal,
                          int nproj, const int* proj_l, const double* proj, int ng,
                          const double* g, double* vloc, double* dvloc, double* vnl) {
  try {
    SpeciesTables s;
    species_from_radial(s, zval, mesh_spacing, nmesh, vlocal, nproj, proj_l, proj, nullptr);
    for (int i = 0; i < ng; i++) {
      double v, dv;
      s.dvlocg(g[i], v, dv);
      if (vloc) vloc[i] = v;
      if (dvloc) dvloc[i] = dv;
      for (int p = 0; p < nproj && vnl; p++) {
        s.dvnlg(p, g[i], v, dv);
        vnl[(size_t)p * ng + i] = v;
      }
    }
    return 0;
  } catch (const Error& e) {
    return e.code;
  } catch (...) {
    return 6;
  }
}

int qbx_host_esr(const double cell[9], int nsp, const int* na, const double* zv,
                 const double* tau, double* esr, double* fion) {
  try {
    std::vector<std::vector<double>> t(nsp), f;
    std::vector<double> z(zv, zv + nsp);
    int off = 0;
    for (int is = 0; is < nsp; is++) {
      t[is].assign(tau + 3 * off, tau + 3 * (off + na[is]));
      off += na[is];
    }
    const double e = esr_energy_forces(cell, t, z, 1.5, f);
    if (esr) *esr = e;
    if (fion) {
      int k = 0;
      for (int is = 0; is < nsp; is++)
        for (double x : f[is]) fion[k++] = x;
    }
    return 0;
  } catch (const Error& e) {
    return e.code;
  } catch (...) {
    return 6;
  }
}

}  // extern "C"
