// Internal declarations of the B200 Kohn-Sham electronic-step library.
//
// One qbx_context owns one Gamma-point SlaterDet on one GPU: the plane-wave
// basis and its staged-FFT stick geometry, species G-space tables, the
// structure factors and projectors of the current atomic positions, and the
// device-resident wavefunctions C, H*C and the stepper history.  Host code
// here builds geometry and tables (the role of the reference's Basis,
// BasisMapping and Species classes); every per-step operation runs on the GPU.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <complex>
#include <iosfwd>
#include <functional>
#include <string>
#include <vector>

namespace qbx {

// ------------------------------------------------------------------ errors
struct Error {
  int code;
  std::string msg;
};

#define QBX_CUDA(call)                                                       \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      throw ::qbx::Error{2, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)
#define QBX_BLAS(call)                                                       \
  do {                                                                       \
    cublasStatus_t s_ = (call);                                              \
    if (s_ != CUBLAS_STATUS_SUCCESS)                                         \
      throw ::qbx::Error{3, std::string(#call) + " failed: " + std::to_string((int)s_)}; \
  } while (0)
#define QBX_SOLVER(call)                                                     \
  do {                                                                       \
    cusolverStatus_t s_ = (call);                                            \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                       \
      throw ::qbx::Error{4, std::string(#call) + " failed: " + std::to_string((int)s_)}; \
  } while (0)
#define QBX_REQUIRE(cond, code, text)                                        \
  do { if (!(cond)) throw ::qbx::Error{code, text}; } while (0)
// after every kernel launch of this library: check it and count it
#define QBX_LAUNCHED(ctx)                                                    \
  do { QBX_CUDA(cudaGetLastError()); (ctx).nlaunch++; } while (0)

// Dynamic shared memory above 48 KB needs a per-kernel opt-in, and that
// attribute is process-wide.  Host threads stepping different systems would
// race if each set the size its own launch needs (a smaller value from one
// thread can land between another's set and launch), so every launch opts in
// to the device maximum less the kernel's static shared memory: the same
// value from every thread.  The need itself is checked here.
template <typename K>
inline void allow_smem(K kernel, size_t need) {
  int dev = 0, optin = 0;
  QBX_CUDA(cudaGetDevice(&dev));
  QBX_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  QBX_CUDA(cudaFuncGetAttributes(&fa, (const void*)kernel));
  const size_t lim = (size_t)optin - fa.sharedSizeBytes;
  QBX_REQUIRE(need <= lim, 20, "kernel shared memory above the device limit");
  QBX_CUDA(cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)lim));
}

// ------------------------------------------------------------ FFT geometry
// A mixed-radix plan for one 1-D length (radices 2,3,4,5,7,8,11).
struct RadixPlan {
  int n = 0;
  int nstage = 0;
  int radix[12] = {0};
};
RadixPlan make_plan(int n);

// Half-sphere basis on the dense grid, ordered rod by rod: rods are the
// z-columns (h,k) of the half sphere in sorted (h,k) order, rod (0,0) first;
// coefficients of one rod are contiguous with l ascending.  Sticks are the
// columns of the full grid that carry data: rod 0 -> stick 0 (holds +l and
// -l), rod r>0 -> stick 2r-1 at (h,k) and stick 2r at (-h,-k).
struct Basis {
  double cell[9];          // rows a0,a1,a2
  double recip[9];         // rows b0,b1,b2 (2 pi inverse transpose)
  double omega = 0;
  double ecut = 0;         // Hartree
  int ng = 0;
  std::vector<int> hkl;    // 3*ng, internal order
  std::vector<double> gx;  // 3*ng (x block, y block, z block)
  std::vector<double> g2, g, gi, g2i;
  int g0 = 0;              // index of G=0 (always 0 in the internal order)
  // rods
  int nrods = 0;
  std::vector<int> rod_h, rod_k, rod_lmin, rod_size, rod_first;
  // grid
  int n0 = 0, n1 = 0, n2 = 0;
  int nvec = 0;                           // sticks = 2*nrods-1
  std::vector<int> stick_x, stick_y;      // grid column of each stick
  int ncol = 0;                           // distinct x columns of sticks
  std::vector<int> stick_col;             // compact column of each stick
  std::vector<int> col_x;                 // grid x of each compact column
  std::vector<int> ip, im;                // grid index of +G and -G
  // complex basis at a k point off Gamma (build_kbasis): gx, g2, g, gi, g2i
  // hold k+G; one stick per rod; im unused
  bool complex_basis = false;
  double kpoint[3] = {0, 0, 0};
  int first = 0;                          // the reference's first local coefficient
};

void build_basis(Basis& b, const double cell[9], double ecut);
void set_grid(Basis& b, int n0, int n1, int n2);
void build_kbasis(Basis& b, const double cell[9], double ecut, const double kpoint[3]);
void set_grid_complex(Basis& b, int n0, int n1, int n2);
bool factorizable(int n);
int fft_size(const double cell[9], double ecut, int dir);
void dense_grid(const double cell[9], double ecut_wf, int np[3]);

// Device copy of the stick geometry used by the staged FFT kernels.
struct DeviceSticks {
  int n0, n1, n2, nrods, nvec, ncol;
  int* rod_first;    // nrods
  int* rod_lmin;     // nrods
  int* rod_size;     // nrods
  int* stick_y;      // nvec
  int* stick_col;    // nvec
  int* col_x;        // ncol
  int* ip;           // ng
  int* im;           // ng
  RadixPlan px, py, pz;
  double2* tw[3];    // exp(+2 pi i k/n) for the x, y, z lengths (owned here,
                     // so contexts of different grids never share tables)
  int* colmap;       // ncol x n1: the stick at (compact column, y), -1 if none
  // widest occupied distance from 0 (mod n) of the stick columns' x, the
  // sticks' y and the rods' z: the pruned plane and z kernels skip the lane
  // registers that only hold points beyond prune_width(n)
  int xw, yw, zw;
};

// Points of a line of length n that the pruned kernels keep: x with
// min(x, n - x) <= prune_width(n).  A wavefunction basis on the grid Qbox
// builds for its density (n >= 4 hmax + 1) always fits.
__host__ __device__ constexpr int prune_width(int n) { return (n - 1) / 4; }

// -------------------------------------------------------------- species
// G-space tables of one species, as the reference's Species holds them after
// initialize() (cubic splines of V_loc(G) and of each projector on a uniform
// G mesh).
struct SpeciesTables {
  double zval = 0, rcps = 1.5;
  int ndft = 0;
  std::vector<double> gspl, vlocg, vlocg2;
  std::vector<int> proj_l;                    // one entry per radial projector
  std::vector<double> proj_d;                 // D matrix (diagonal, per l)
  std::vector<std::vector<double>> vnlg, vnlg2;
  int nlm() const {
    int n = 0;
    for (int l : proj_l) n += 2 * l + 1;
    return n;
  }
  double eself() const;
  void dvlocg(double g, double& v, double& dv) const;
  void dvnlg(int iop, double g, double& v, double& dv) const;
  double rhopsg(double g) const;
};
void species_from_radial(SpeciesTables& s, int zval, double mesh_spacing,
                         int nmesh, const double* vlocal, int nproj,
                         const int* proj_l, const double* proj,
                         const double* proj_d);

double esr_energy_forces(const double cell[9],
                         const std::vector<std::vector<double>>& tau,
                         const std::vector<double>& zv, double rcps,
                         std::vector<std::vector<double>>& f, double* sigma = nullptr);

// ---------------------------------------------------------------- context
enum Precision { FP64 = 0, MIXED = 1 };

// CUDA-event timing of tagged regions on the context's stream.  When
// enabled, each region records an event pair; qbx_profile_get() resolves the
// pairs into per-tag total milliseconds and counts.
struct Profiler {
  bool on = false;
  std::vector<std::string> names;
  std::vector<double> ms;
  std::vector<long> count;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> pool;
  int tag(const std::string& n) {
    for (size_t i = 0; i < names.size(); i++)
      if (names[i] == n) return (int)i;
    names.push_back(n); ms.push_back(0.0); count.push_back(0);
    return (int)names.size() - 1;
  }
  cudaEvent_t get() {
    if (pool.empty()) {
      cudaEvent_t e;
      QBX_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void resolve() {
    for (auto& p : pending) {
      float t = 0.f;
      QBX_CUDA(cudaEventElapsedTime(&t, p.second.first, p.second.second));
      ms[p.first] += t;
      count[p.first] += 1;
      pool.push_back(p.second.first);
      pool.push_back(p.second.second);
    }
    pending.clear();
  }
  void reset() {
    resolve();
    for (auto& m : ms) m = 0.0;
    for (auto& c : count) c = 0;
  }
};

// Device scalar slots.  Every reduction of the electronic step writes its
// sums into a fixed slot of ctx.d_scalars and nothing reads them back while
// the step runs; the host copies all slots once (readback) and derives the
// energies from that copy (finish_*).  With no host synchronisation inside,
// a step can be captured as one CUDA graph.
enum : int {
  SLOT_CHARGE = 0,     // sum_r rho(r)
  SLOT_EXC = 1,        // sum_r e_xc(r), sum_r rho v1 (PBE), sum_r rho v_xc
  SLOT_EPS_EH = 4,     // sum rho*(G) vion(G); sum |G|^-2 times |rho_tot|^2,
                       // |rho_e|^2, |rho_ps|^2 (total, electronic, pseudocharge)
  SLOT_EKIN = 8,
  SLOT_ENL = 9,
  SLOT_EIG = 10,
  SLOT_ANDERSON = 11,  // the two sums of the Anderson theta
  SLOT_THETA = 13,     // theta used by the last PSDA step
  SLOT_FROB = 14,      // ||I - x^T x||_F^2 of the current polar iterate
  SLOT_STRESS = 16,    // 30 sums of the stress tensor parts
  SLOT_SCRATCH = 56,   // one-off sums
  SLOT_MIX = 64,       // the normal matrix and right-hand side of the charge mixer
  kSlots = 128
};
// Device status words of a step (int): solver info codes, the polar
// iteration count and the tcgen05 wait-timeout flag.
enum : int {
  ST_INFO_GRAM = 0,
  ST_INFO_ORTHO = 1,
  ST_INFO_POLAR = 2,
  ST_POLAR_ITERS = 3,
  ST_TC_ERR = 4,
  kStatus = 8
};

// One captured electronic step (PSDA, with or without forces, with or
// without the Anderson extrapolation): an instantiated graph and the
// number of this library's kernels it holds outside the polar loop.
struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  long id = 0;                   // unique per capture (process-wide), 0 = none
  long nkernels = 0;
  int uses = 0;        // eager runs of this configuration before capture
};

// One graph holding the steps of several contexts as parallel branches
// (qbx_scf_step_batch, one multi-stream capture), cached on the first
// context of the batch and rebuilt when the members' captured steps change.
struct BatchGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<long> ids;         // StepGraph ids of the members, in order
  bool failed = false;           // instantiation refused: launch per context
};

// One k point off Gamma (Wavefunction::add_kpoint): its complex basis and
// stick geometry, the coefficients and H*psi (ngw x nst complex, column-major
// like ComplexMatrix), the PSDA history and the projector columns at k+G.
struct KPointSet {
  double k[3] = {0, 0, 0};   // units of the reciprocal vectors
  double weight = 0;
  Basis kb;
  DeviceSticks dks{};
  double* d_c = nullptr;       // 2*ngw*nst
  double* d_hc = nullptr;
  double* d_c_last = nullptr;
  double* d_dc_last = nullptr;
  double* d_ctmp = nullptr;
  double* d_g2 = nullptr;      // |k+G|^2
  double* d_q = nullptr;       // k+G, x, y and z blocks
  double* d_twnl = nullptr;    // projector forms at k+G
  double* d_anl = nullptr;     // 2*ngw*nproj
  double* d_w2 = nullptr;      // weight*occ/Omega twice per band (plane kernel weights)
  double* d_prec = nullptr;    // nst per-band kinetic energies
  bool anl_ready = false;
  double theta = 0;
};

struct Context {
  int device = 0;
  int precision = FP64;
  std::string last_error;
  cudaStream_t stream = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  bool have_cell = false;

  Basis wb, vb;                 // wavefunction basis, density basis (4 ecut)
  DeviceSticks dws{}, dvs{};
  DeviceSticks dwg{};           // the wavefunction basis on its own FFT grid (sample files)
  bool have_wgrid = false;
  std::string xc = "LDA";

  // species and atoms
  std::vector<SpeciesTables> species;
  std::vector<std::vector<double>> tau;   // per species, 3*na
  double esr = 0, eself = 0;
  std::vector<std::vector<double>> fion_esr;
  int nproj = 0;                // total projector columns (sum nlm*na)
  std::vector<int> proj_species, proj_atom, proj_lm;   // per column
  std::vector<double> proj_dfac;                       // D per column

  // wavefunctions
  int nst = 0;
  std::vector<double> occ;
  bool extrapolate = false;
  int wf_dyn = 0;               // 0: PSDA, 1: JD (the reference's wf_dyn)
  double* d_jd_h = nullptr;     // 2nst x 2nst projected Hamiltonian
  double* d_jd_w = nullptr;     // its eigenvalues
  double* d_jd_work = nullptr;  // syevd workspace
  int jd_lwork = 0;

  // device buffers (double unless noted)
  double* d_gx_w = nullptr;     // 3*ngw
  double* d_g2_w = nullptr;     // ngw
  double* d_gx_v = nullptr;     // 3*ngv
  double* d_g2i_v = nullptr;    // ngv
  double* d_c = nullptr;        // 2*ngw*nst  (complex, band-major)
  double* d_hc = nullptr;
  double* d_c_last = nullptr;
  double* d_dc_last = nullptr;
  double* d_ctmp = nullptr;     // scratch copy of C
  double* d_xsd = nullptr;      // a caller's SlaterDet (class-level entry points), lazy
  double* d_xgrid = nullptr;    // a caller's grid function (class-level entry points), lazy
  double* d_occ = nullptr;      // nst
  double* d_anl = nullptr;      // 2*ngw*nproj  (complex projectors x phase)
  double* d_fnl = nullptr;      // nproj*nst
  double* d_dfnl = nullptr;     // nproj*nst
  double* d_pdfac = nullptr;    // nproj
  int* d_patom = nullptr;       // nproj (global atom index)
  double* d_rhor = nullptr;     // N
  double* d_vr = nullptr;       // N
  double* d_vxc = nullptr;      // N
  double* d_exc = nullptr;      // N (energy density scratch)
  double* d_vx2 = nullptr;      // N (PBE vxc2)
  double* d_grad = nullptr;     // 3N
  double* d_rhog = nullptr;     // 2*ngv (complex)
  double* d_vion = nullptr;     // 2*ngv
  double* d_rhops = nullptr;    // 2*ngv (sum of S*rhops)
  double* d_vtmp_g = nullptr;   // 2*ngv scratch
  double* d_vtmp_g2 = nullptr;  // 2*ngv scratch
  double* d_xc_g = nullptr;     // 3 x 2*ngv: the GGA's density-basis coefficients
  double* d_sfac = nullptr;     // 2*ngv*nsp
  double* d_vps = nullptr;      // ngv*nsp
  double* d_rhops_sp = nullptr; // ngv*nsp
  void* d_grid = nullptr;       // N complex (double2) scratch for vbasis FFTs
  void* d_zbuf = nullptr;       // staged FFT stick buffer
  size_t zbuf_bytes = 0;
  int pair_batch = 0;
  double* d_nn = nullptr;       // nst*nst matrices (4 of them)
  double* d_nn2 = nullptr;
  double* d_nn3 = nullptr;
  double* d_nn4 = nullptr;
  double* d_nn5 = nullptr;      // n x n: L^-1 of ortho_align's overlap (mixed path)
  int* d_ipiv = nullptr;
  int* d_info = nullptr;
  double* d_solver_work = nullptr;
  int solver_lwork = 0;
  double* d_red = nullptr;      // reduction partials
  double* d_scalars = nullptr;  // kSlots scalar slots, then the density weights
  double* h_scalars = nullptr;  // pinned host copy of the slots
  int* d_status = nullptr;      // kStatus status words
  int* h_status = nullptr;      // pinned host copy
  double* h_fion = nullptr;     // pinned host copy of d_fion
  double* d_prec = nullptr;     // nst ekin per band
  double* d_fion = nullptr;     // 3*natoms

  // energies of the last evaluation
  double ekin = 0, eps = 0, enl = 0, ehart = 0, exc = 0, ecoul = 0,
         etotal = 0, total_charge = 0, eigsum = 0, theta = 0;
  std::vector<double> fion;     // 3*natoms, species-major like the reference

  // stress (EnergyFunctional::energy with compute_stress)
  double sigma_esr[6] = {0, 0, 0, 0, 0, 0};
  double sigma[6] = {0, 0, 0, 0, 0, 0};
  double sigma_parts[36] = {0};  // ekin, eps, enl, ehart, exc, esr (6 each)
  bool have_stress = false;
  double xc_rhov1 = 0;          // sum_r rho v1 of the last PBE update (stress)
  double dxc = 0, ehart_e = 0, ehart_p = 0;   // Harris-Foulkes terms of update_vhxc
  // charge mixing of the SCF loop with nite > 0 (scf.cu)
  double* d_rhog_in = nullptr;  // 2*ngv: the mixed rho(G)
  double* d_mix = nullptr;      // 2*(ndim+1) vectors of 2*ngv: Anderson x and f history
  double* d_wmix = nullptr;     // 2*ngv: least-squares weights, Kerker weights
  int mix_ndim = -1;            // history length the buffers were made for
  double mix_rcut = -1.0;
  double* d_dvps = nullptr;     // ngv*nsp: dV_loc/dG / Omega per species
  double* d_vnl = nullptr;      // nrad*ngw: radial projector V_nl(|G|)
  double* d_dvnl = nullptr;     // nrad*ngw: dV_nl/dG
  int* d_pcol = nullptr;        // 4*nproj: (l, m, radial row, atom) per column
  double* d_tau_all = nullptr;  // 3*natoms
  double* d_phase_tab = nullptr;   // per atom exp(-i 2 pi h u_j) tables (structure factors)
  size_t phase_tab_bytes = 0;
  double* d_fpart = nullptr;    // slice partials of the local forces (3 natoms x 16)
  size_t fpart_elems = 0;
  double* d_twnl = nullptr;     // projector forms Y_lm V_nl, one ngw row per (species, l, m)
  double* d_astress = nullptr;  // 2*ngw*nproj: a strain-derivative projector block
  void* sa_hi = nullptr;        // its BF16 split (mixed path)
  void* sa_lo = nullptr;

  // mixed precision: BF16 hi/lo splits of the GEMM operands
  int gemm_backend = 1;         // 0: cuBLAS BF16 products, 1: own tcgen05 kernel
  int tc_chunk = 2;             // tcgen05 GEMM: K blocks per TMEM chain of the hi*hi term
  int tc_corr_mul = 8;          // tcgen05 GEMM: hi*lo + lo*hi chains this many times longer,
                                // in accumulators of their own (0: in the hi*hi chain)
  int tc_epw = 8;               // tcgen05 GEMM: epilogue warps (4 or 8)
  int tc_pair = 2;              // tcgen05 GEMM on CTA pairs (cta_group::2): 0 off (one CTA per
                                // 128 x 128 tile), 1 256 x 128 tiles, 2 256 x 256 tiles
  int tc_pair_epw = 16;         // epilogue warps of the 256 x 256 pair tiles (8 or 16)
  int tc_tf32_mn = 1;           // TF32 tall updates read the plain split MN-major (else a
                                // transposed split)
  int step_fuse = 1;            // mixed PSDA step: band energies of the preconditioner, the
                                // eigenvalue sum and C's splits made inside neighbouring
                                // passes (0: each in a pass of its own)

  // band pairs split over GPUs (qbx_set_band_shard): this GPU's rank among
  // shard_n, and the NCCL communicator (ncclComm_t) of the group
  int shard_rank = 0, shard_n = 1;
  void* shard_comm = nullptr;
  void* d_acc32 = nullptr;      // FP32 product accumulator
  double* d_colred = nullptr;   // per-column partial sums of the fused split kernels
  size_t colred_elems = 0;
  size_t acc32_elems = 0;
  void* cs_hi[2] = {nullptr, nullptr};   // splits of C (0: at energy, 1: after the step)
  void* cs_lo[2] = {nullptr, nullptr};
  void* hs_hi = nullptr;        // split of H C
  void* hs_lo = nullptr;
  void* as_hi = nullptr;        // split of the projectors
  void* as_lo = nullptr;
  void* ss_hi = nullptr;        // split of a small matrix (fnl, A, X)
  void* ss_lo = nullptr;
  int ldp = 0;                  // padded leading dimension of the K-row splits
  float* c32 = nullptr;         // TF32 hi/lo split of C (tall updates)
  float* c32lo = nullptr;
  float* d_vr32 = nullptr;      // FP32 copy of V(r) for the mixed H*psi pass
  void* d_zfast = nullptr;      // stick buffer of the specialised staged FFTs
  size_t zfast_bytes = 0;
  int fast_batch = 0;           // band pairs per launch (0: as many as fit)
  int fast_rods = 16;           // rods per CTA of the z kernels
  int fast_warps = 16;          // warps per CTA of the plane kernel (at most)
  int fast_vpsi_shape = 0;      // FP32 H*psi plane CTA shape (0, 1, 2)
  int fast_lane_shape = 4;      // FP32 register-lane plane kernel shape (5: sticks through
                                // the column map), -1 = off
  int fast_density_lane_shape = 3;  // its density shape (2, 3; 5 half planes; 6 sticks
                                    // read through the column map; 7 TMEM accumulator;
                                    // 8 next pair's sticks queued with cp.async)
  int fast_chunks = 8;          // CTAs per plane in the density pass
  int fast_fwd_ppc = 2;         // band pairs per CTA of the H*psi plane kernel from psi(r)
  int fast_fwd_staged = 1;      // that kernel with its rows staged by cp.async
  int fast_prune = 1;           // FP32 lane kernels skip the points beyond the sphere
                                // (prune_width) where the basis allows it
  int fast_zlane = 1;           // FP32 z sticks in register lanes (0: warp per stick;
                                // 2: backward uncapped; 3: forward only)
  bool fast_fft = true;         // use the specialised kernels when compiled
  float* a32 = nullptr;         // TF32 hi/lo split of the projectors
  float* a32lo = nullptr;
  float* s32 = nullptr;         // TF32 hi/lo split of a small matrix
  float* s32lo = nullptr;
  int tall_kind = 1;            // split kind of the rotation C (I - X): TF32 by default
  int tall_kind_hc = 0;         // split kind of the H*C updates A_nl F and C A: BF16
  void* at_hi = nullptr;        // split of A_nl^T (projectors contiguous), ld tall_ld(nproj)
  void* at_lo = nullptr;
  void* ct_hi = nullptr;        // split of C^T (bands contiguous), ld tall_ld(nst)
  void* ct_lo = nullptr;
  void* tm_hi = nullptr;        // split of the small right-hand matrix, ld tall_ld(rows)
  void* tm_lo = nullptr;
  // leading dimension of a split of the given kind (16-byte rows)
  static int tall_ld_of(int kind, int n) { return kind == 1 ? (n + 3) / 4 * 4 : (n + 7) / 8 * 8; }
  int tall_ld(int n) const { return tall_ld_of(tall_kind, n); }
  void* d_tc_ws = nullptr;      // split-K partials of the tcgen05 GEMM
  size_t tc_ws_elems = 0;
  long nlaunch = 0;              // kernels of this library launched so far
  Profiler prof;

  // graph-captured steps (qbx_set_step_graph)
  bool step_graph = false;
  bool capturing = false;        // a step is being captured on `stream`
  StepGraph graphs[4];           // by (extrapolate, forces)
  BatchGraph batch;              // batch graph led by this context
  bool batch_single_graph = false;   // QBX_BATCH_GRAPH=1: batch steps as one graph
  cudaStream_t side[2] = {nullptr, nullptr};   // capture of conditional bodies
  void* d_blas_ws = nullptr;     // cuBLAS workspace bound with every stream
  size_t blas_ws_bytes = 0;
  std::string graph_note;        // why the last capture was abandoned, if it was
  long graph_launches = 0;       // captured steps launched so far
  long batch_launches = 0;       // batch graphs launched with this context leading
  int polar_iters = 0;           // iterations of the last eager polar
  double* d_wfv = nullptr;       // wavefunction velocity of the MD extrapolation
  // psi(r) of every band pair kept in HBM (FP32) from the density pass to
  // the H*psi pass of the same step: the step functions set psir_store
  // around update_density and psir_use around energy
  float2* d_psir = nullptr;
  size_t psir_bytes = 0;
  int psir_mode = -1;            // -1 auto (mixed precision, if it fits), 0 off, 1 on
  bool psir_store = false, psir_use = false, psir_valid = false;
  const double* psir_src = nullptr;   // the coefficients psi(r) was made from
  // streamed SlaterDet (qbx_stream_in / qbx_scf_step_async / qbx_stream_out):
  // two copy streams, the staging buffers of one step's input and result,
  // and the events that order them against the compute stream
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_in = nullptr, ev_cin_free = nullptr, ev_step = nullptr, ev_out = nullptr;
  double* d_cin = nullptr;
  double* d_cout = nullptr;
  bool in_pending = false;       // an upload not yet consumed by a step
  bool finish_pending = false;   // a captured step whose host finish is deferred
  double last_energies[16] = {0};
  // k points off Gamma; when set, the electronic step runs on them instead
  // of the Gamma coefficients
  std::vector<KPointSet> kpts;
  bool kpts_extrapolate = false;
  double* d_fnlk = nullptr;      // 2*nproj*nst complex projections of one k point
  double* d_znn = nullptr;       // 6 complex nst x nst matrices
  double* d_zwork = nullptr;     // cuSOLVER workspace of the complex factorisations
  int zwork_len = 0;             // its length in complex elements
  int* d_zipiv = nullptr;        // nst pivots + 1 info word

  size_t N() const { return (size_t)vb.n0 * vb.n1 * vb.n2; }
};

// Records the tagged region [construction, destruction) on ctx.stream when
// the profiler is on.
struct ProfScope {
  Context& c;
  int t = -1;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(Context& ctx, const char* name) : c(ctx) {
    if (!c.prof.on) return;
    t = c.prof.tag(name);
    a = c.prof.get();
    b = c.prof.get();
    QBX_CUDA(cudaEventRecord(a, c.stream));
  }
  ~ProfScope() {
    if (t < 0) return;
    if (cudaEventRecord(b, c.stream) == cudaSuccess)
      c.prof.pending.push_back({t, {a, b}});
  }
};

// device memory helpers
template <typename T>
inline T* dalloc(size_t n) {
  if (n == 0) return nullptr;
  void* p = nullptr;
  QBX_CUDA(cudaMalloc(&p, n * sizeof(T)));
  return (T*)p;
}
template <typename T>
inline void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}
// Host-to-device copy that has fully landed when it returns.  Kernels run on
// a non-blocking stream, which does not order itself after the legacy
// stream's copies, and a pageable cudaMemcpy may return before its DMA ends;
// the device synchronisation closes both gaps.  Setup paths only.
inline void h2d_sync(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  QBX_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  QBX_CUDA(cudaDeviceSynchronize());
}
template <typename T>
inline T* dupload(const std::vector<T>& v) {
  T* p = dalloc<T>(v.size());
  h2d_sync(p, v.data(), v.size() * sizeof(T));
  return p;
}

// ---------------------------------------------------- kernel launchers
// staged wavefunction FFTs (fft.cu)
void upload_sticks(DeviceSticks& d, const Basis& b);
void free_sticks(DeviceSticks& d);
// rho(r) += sum_n occ_n/omega |psi_n(r)|^2 over all bands of c
void launch_density(Context& ctx, const double* c, double* rho);
// hc = 1/2 |G|^2 c + FFT_fwd(v FFT_bwd(c))  (hc overwritten)
void launch_vpsi(Context& ctx, const double* c, const double* v, double* hc);
// vbasis transforms on the full grid
void vb_backward(Context& ctx, const double* coef, double* real_out);   // real part
void vb_forward_real(Context& ctx, const double* f, double scale, double* coef);
// two real fields in one complex transform: out0 + i out1 from the
// coefficients a and b (both of real fields, half sphere)
void vb_backward_pair(Context& ctx, const double* a, const double* b, double* out0, double* out1);
// the coefficients of f0 w and f1 w (f1 may be null) from one complex
// transform, with the 1/N of the forward transform
void vb_forward_real_pair(Context& ctx, const double* f0, const double* f1, const double* w,
                          double* c0, double* c1);
// wavefunction-basis single transforms through the full-grid path (tests)
void wb_backward_pair(Context& ctx, const double* c1, const double* c2, double* grid_out);

// staged-FFT launch configuration by timing on the context's own data
void autotune_fft(Context& ctx, std::vector<std::pair<std::string, double>>* log);

// occ_n / Omega per band (device), used by the density kernels
double* density_weights(Context& ctx);

// pointwise kernels (kernels.cu)
void launch_sum(Context& ctx, const double* x, size_t n, int slot);   // slot = sum x
void launch_xc(Context& ctx);                  // fills d_vxc; SLOT_EXC
void launch_vhxc_gspace(Context& ctx);         // SLOT_EPS_EH, vlocal_g
void launch_setup_atoms(Context& ctx);         // sfac, vion, rhops, anl
void launch_ekin(Context& ctx);                // SLOT_EKIN
void launch_eigsum(Context& ctx);              // SLOT_EIG
void launch_precond_update(Context& ctx);      // d_prec
// residual -> step; SLOT_THETA.  split_c: also C's cleanup and the splits
// that ortho_align reads when ortho_splits_both (one pass)
void launch_psda_elementwise(Context& ctx, bool split_c = false);
void launch_precondition_into(Context& ctx, const double* r, double* z);   // z = -K r
void launch_cleanup(Context& ctx, double* c);  // Im c(G=0) = 0
void launch_rank1_fix(Context& ctx, double* m, int ldm, const double* x, int ldx,
                      const double* y, int ldy, int nrow, int ncol, double alpha,
                      bool lower_only);
void launch_enl(Context& ctx);                  // SLOT_ENL; fnl <- DF/omega
void launch_local_forces(Context& ctx, double* fion);
void launch_nl_forces(Context& ctx, double* fion);
// stress tensor of the state of the last energy(): SLOT_STRESS; then
// finish_stress gives ctx.sigma, ctx.sigma_parts
void compute_stress(Context& ctx);
// band-pair sharding (shard.cu): this GPU's pairs [lo, hi); the sum of a
// device array over the GPUs; the gather of every GPU's bands of a
// band-major K x nst block; the communicator's release
void shard_pairs(const Context& ctx, int& lo, int& hi);
void shard_sum(Context& ctx, double* x, size_t n);
void shard_gather_bands(Context& ctx, double* x);
void shard_release(Context& ctx);
void compute_stress_nl(Context& ctx);            // the nonlocal part alone (SS_ENL slots)
void nl_stress_part(const Context& ctx, double enl, double* sigma_enl);   // after readback
// NonLocalPotential::energy on its own: E_nl into its slot and, with hpsi,
// the nonlocal part of H*C written to out (device, K x nst)
void nonlocal_only(Context& ctx, bool hpsi, double* out);
// Wavefunction::diag: eigenvalues of C^T H C into w (device, nst); with
// eigvec C <- C Z and H*C <- the previous C
void diag(Context& ctx, bool eigvec, double* w);
void launch_identity_axpy(Context& ctx, double* t, const double* q, int n,
                          double alpha);       // t = I + alpha*q
void launch_symmetrize_lower(Context& ctx, double* q, int n);
void launch_avg_transpose(Context& ctx, double* x, const double* t, int n);
void launch_frob2(Context& ctx, const double* q, int n);   // SLOT_FROB = ||q||_F^2
void launch_sumsq(Context& ctx, const double* x, size_t len, int slot);   // sum of x_i^2
// Conditional graph nodes of a step being captured (step.cu): the graph
// captured on s; a conditional node of the given type after s's current
// dependencies (returns its bodies); f captured into body on stream s; the
// polar loop's decision from SLOT_FROB (Bjorck-Bowie branch when the norm
// is below one; another iteration while above tol and under maxiter).
cudaGraph_t capture_graph(cudaStream_t s);
cudaGraph_t* add_conditional(cudaStream_t s, cudaGraphConditionalHandle h,
                             cudaGraphConditionalNodeType type, unsigned size);
void capture_body(Context& ctx, cudaGraph_t body, cudaStream_t s, const std::function<void()>& f);
void launch_polar_decide(Context& ctx, double tol, int maxiter, int* iters,
                         cudaGraphConditionalHandle loop, cudaGraphConditionalHandle branch);

// ------------------------------------------------ scalars of a step (scalars.cu)
// Copies the slots and status words (and d_fion when `fion`) to their pinned
// host mirrors on ctx.stream; no synchronisation (graph-capturable).
void enqueue_readback(Context& ctx, bool fion);
// enqueue_readback + wait for ctx.stream
void readback(Context& ctx, bool fion);
// one slot read now (synchronising; eager paths only)
double read_slot(Context& ctx, int slot);
// host values derived from the mirrors
void finish_density(Context& ctx);   // total_charge
void finish_vhxc(Context& ctx);      // exc, xc_rhov1, eps, ehart
void finish_energy(Context& ctx, bool forces);   // ekin, enl, ecoul, etotal (+ fion)
void finish_eigsum(Context& ctx);    // eigsum
void finish_theta(Context& ctx);     // theta
void finish_stress(Context& ctx);    // sigma, sigma_parts
// throws the first nonzero status word as an error
void check_status(Context& ctx);
// binds cuBLAS (with the context's workspace) and cuSOLVER to stream s
void bind_stream(Context& ctx, cudaStream_t s);

// ------------------------------------------------ the step and its callers
void gram(Context& ctx, bool split_overlap = false);
// c_split_done: the caller has cleaned up C and written the splits that
// ortho_splits_both names (launch_psda_elementwise with split_c)
void ortho_align(Context& ctx, bool c_split_done = false);
// ortho_align reads C's BF16 and TF32 splits, made in one pass
bool ortho_splits_both(const Context& ctx);
void update_density(Context& ctx);
void update_vhxc(Context& ctx);
void energy(Context& ctx, bool hpsi, bool forces);
// psda_update's fusions, for callers that ran energy() on the same C just
// before: PSDA_PREC_FROM_ENERGY takes the preconditioner's band energies
// from energy()'s split pass (mixed path), PSDA_EIGSUM forms the eigenvalue
// sum (SLOT_EIG) in the split of H C (mixed path; launch_eigsum otherwise)
enum : unsigned { PSDA_PREC_FROM_ENERGY = 1u, PSDA_EIGSUM = 2u };
void psda_update(Context& ctx, unsigned fuse = 0);
// energy()'s mixed path forms the preconditioner's band energies too
bool energy_forms_prec(const Context& ctx);
void jd_update(Context& ctx);
void polar_factor(Context& ctx, double* x, double tol, int maxiter);
// Li = L^-1 of a lower-triangular n x n L (ld n), blocked for n = 32 x a power
// of two (work: n * n / 4 doubles), else a triangular solve of I
bool lower_inverse_blocked(int n);
void lower_inverse(Context& ctx, const double* L, int n, double* Li, double* work);
int polar_entry(Context& ctx, double* x, double tol, int maxiter, bool graph);
// one electronic step (captured graph or eager), energies/fion as qbx_scf_step
void scf_step_any(Context& c, bool want_f, bool want_s, double* energies, double* fion);
void align_to_c(Context& ctx, double* cv);   // SlaterDet::align of cv to C
void lowdin(Context& ctx);                     // SlaterDet::lowdin of C
// SCF loop with charge mixing (scf.cu); energies as arrays of the
// iterations (see qbx_scf_run)
void scf_run(Context& c, int nitscf, int nite, double mix_coeff, double mix_rcut, int mix_ndim,
             double scf_tol, double* etotal_int, double* eigsum, int* nite_done, int* nitscf_done);
void free_mix(Context& c);
// sample-file wavefunctions (sample_io.cpp)
void write_wavefunction(Context& c, std::ostream& os);
void read_wavefunction(Context& c, const std::string& text);
void wfgrid_backward(Context& ctx, const DeviceSticks& d, int ng, const double* c, double* f);
void upload_grid_map(DeviceSticks& d, int n0, int n1, int n2, const std::vector<int>& ip,
                     const std::vector<int>& im);
void basis_ft_backward(Context& ctx, const DeviceSticks& d, int ng, bool real_basis,
                       const double* c1, const double* c2, double* grid);
void basis_ft_forward(Context& ctx, const DeviceSticks& d, int ng, bool real_basis, double* grid,
                      double* c1, double* c2);
void wfgrid_forward(Context& ctx, const DeviceSticks& d, int ng, const double* f, double* c);
// molecular dynamics (md.cu)
void move_atoms(Context& c, const double* tau);
// k points off Gamma (kpoint.cu)
void set_kpoints(Context& ctx, int nk, const double* k, const double* w);
void free_kpoints(Context& ctx);
void kpoints_atoms_changed(Context& ctx);
void gram_k(Context& ctx);
void update_density_k(Context& ctx);
void energy_k(Context& ctx, bool hpsi);
void eigsum_k(Context& ctx);
void psda_update_k(Context& ctx);
std::vector<double> twnl_rows(const Context& ctx, const Basis& b);
void build_anl(Context& ctx, const double* d_q, int ngw, const double* d_twnl, double* d_anl);
void launch_density_k(Context& ctx, KPointSet& kp, double* rho);
void launch_vpsi_k(Context& ctx, KPointSet& kp, const double* v);
void md_run(Context& c, int niter, int nitscf, double dt, const double* mass_amu, double* vel,
            double* tau_out, double* ionic, double* scf);

// split-precision products (split_gemm.cu, tc_gemm.cu)
void split_bf16(Context& ctx, const double* x, size_t n, void* hi, void* lo);
void overlap_diag_f64(Context& ctx, const double* c, int K, int n, double* S);
// C = alpha * op(A) op(B) + beta * C, C column-major with ld m
// lower: only the tiles holding the lower triangle of a square C are
// formed (the tcgen05 backend; the others form all of C)
void split_gemm(Context& ctx, bool ta, bool tb, int m, int n, int k, double alpha,
                const void* ahi, const void* alo, int lda, const void* bhi, const void* blo,
                int ldb, double beta, double* C, bool lower = false);
bool tc_gemm_supported(const Context& ctx, bool ta, bool tb, int m, int n, int k);
void tc_split_gemm(Context& ctx, bool ta, bool tb, int m, int n, int k, double alpha,
                   const void* ahi, const void* alo, int lda, const void* bhi, const void* blo,
                   int ldb, double beta, double* C, bool lower = false);
int tc_check_error(Context& ctx);   // nonzero if a tcgen05 GEMM wait ran out
void split_bf16_2d(Context& ctx, const double* x, int rows, int cols, int ldx, void* hi, void* lo,
                   int ldp);
// both splits of one block in one pass: BF16 hi/lo (ld ldb, padding rows
// zero) and TF32 hi/lo (ld ldt)
void split_bf16_tf32(Context& ctx, const double* x, int rows, int cols, int ldx, void* bhi,
                     void* blo, int ldb, float* thi, float* tlo, int ldt);
// the BF16 split of a wavefunction block (rows = 2 ngw) with the kinetic sum
// sum_n occ_n sum_G g2(G) |c_n(G)|^2 of the same pass into *out; with prec,
// also each band's kinetic energy for the preconditioner into prec[cols]
void split_bf16_ekin(Context& ctx, const double* x, int rows, int cols, int ldx, void* hi,
                     void* lo, int ldp, const double* g2, const double* occ, double* out,
                     double* prec = nullptr);
// the BF16 split of a wavefunction block x (rows = 2 ngw) with the sum over
// its columns of 2 Re <x_n, y_n> - x_n(0) y_n(0) (y of x's layout) into *out
void split_bf16_dot(Context& ctx, const double* x, const double* y, int rows, int cols, int ldx,
                    void* hi, void* lo, int ldp, double* out);
// CTAs per column of the split kernels over span rows (at most 64): the
// number of column partials that the finishing kernels add
int split_blocks_per_column(int span);
// diag(S) = 2 C^T C - c0 c0^T on the diagonal, exact in FP64, from the
// column sums of the last split_bf16_tf32 of c
void overlap_diag_from_split(Context& ctx, const double* c, int K, int n, int ldp, double* S);
void split_tf32(Context& ctx, const double* x, int rows, int cols, int ldx, float* hi, float* lo,
                int ldy);
void tf32x3_gemm_nn(Context& ctx, int m, int n, int k, double alpha, const float* Ahi,
                    const float* Alo, int lda, const float* Bhi, const float* Blo, int ldb,
                    double beta, double* C, int ldc);
inline int pad4(int n) { return (n + 3) / 4 * 4; }
inline int pad8(int n) { return (n + 7) / 8 * 8; }
// split kinds of the tall updates: BF16 hi/lo (kind::f16) or TF32 hi/lo
// (kind::tf32, stored as FP32)
enum { TALL_BF16 = 0, TALL_TF32 = 1 };
// x as hi/lo of the given kind, leading dimension ldy (BF16: padding rows zero)
void split_plain(Context& ctx, int kind, const double* x, int rows, int cols, int ldx, void* hi,
                 void* lo, int ldy);
// x^T as hi/lo of the given kind: x rows x cols (ld ldx) -> cols x rows (ld ldy)
void split_t(Context& ctx, int kind, const double* x, int rows, int cols, int ldx, void* hi,
             void* lo, int ldy);
// C (m x n, ld ldc) = alpha A^T B + beta C with hi/lo splits A (k x m, ld
// lda) and B (k x n, ld ldb) of the given kind, through the tcgen05 kernel
void tc_gemm_kind_tn(Context& ctx, int kind, int m, int n, int k, double alpha, const void* ahi,
                     const void* alo, int lda, const void* bhi, const void* blo, int ldb,
                     double beta, double* C, int ldc);
// C (m x n) = alpha * A B + beta * C with A given as its plain split (m
// contiguous, lda between columns) and B (k x n) K-major: the tall update
// without a transposed copy of A (CTA pairs on 256 x 256 tiles)
void tc_gemm_kind_nn_mn(Context& ctx, int kind, int m, int n, int k, double alpha, const void* ahi,
                        const void* alo, int lda, const void* bhi, const void* blo, int ldb,
                        double beta, double* C, int ldc);
void tc_tf32_gemm_tn(Context& ctx, int m, int n, int k, double alpha, const float* ahi,
                     const float* alo, int lda, const float* bhi, const float* blo, int ldb,
                     double beta, double* C, int ldc);
void alloc_mixed(Context& ctx);
void split_projectors(Context& ctx);   // after the projectors change (mixed)
void free_mixed(Context& ctx);

}  // namespace qbx

namespace qbx {
// Density pass with caller-supplied stick buffer and twiddle tables
// (exp(+2 pi i k/n) for the x, y and z lengths); adds into rho.
size_t density_stick_bytes_per_pair(const Context& ctx);
void density_with_buffers(Context& ctx, const double* c, int nst, const double* w, double* rho,
                          void* zbuf, size_t zbuf_bytes, const double2* twx, const double2* twy,
                          const double2* twz);
}  // namespace qbx
