/*
 * qbx.h - C ABI of the B200 Kohn-Sham electronic step.
 *
 * One qbx_context holds one Gamma-point Slater determinant on one GPU (the
 * reference's Context collapsed to one process).  The entry points mirror
 * the reference Qbox classes on the electronic-step path; each names the
 * reference interface it replaces.  All arrays are host pointers unless the
 * name says otherwise; all sizes are element counts.  Every call returns 0
 * on success or a positive error code; qbx_last_error() gives the message.
 *
 * Conventions (as in the reference):
 *  - units are Hartree atomic units; ecut is in Hartree (the reference's
 *    `set ecut` value in Rydberg divided by 2, src/Ecut.h:40-50);
 *  - coefficients are complex doubles (re, im interleaved), band-major:
 *    c[2*(n*ngw + ig) + {0,1}], ig over the half sphere of G vectors;
 *  - the default coefficient order is sorted Miller index (h,k,l), the order
 *    returned by qbx_basis_miller(); any other order can be used by passing
 *    the caller's Miller indices to qbx_set_coeff_order();
 *  - real-space grids are np0*np1*np2 doubles, x fastest
 *    (src/BasisMapping.cpp:206-216);
 *  - energies[QBX_NENERGY] = { ekin, eps, enl, ehart, ecoul, exc, esr, eself,
 *    etotal, eigenvalue_sum, total_charge, theta }.
 */
#ifndef QBX_H
#define QBX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qbx_context qbx_context;

#define QBX_FP64 0   /* FP64 FFTs and FP64 GEMMs                        */
#define QBX_MIXED 1  /* FP32 FFTs; FP64 storage, reductions, Cholesky   */
#define QBX_NENERGY 12

int qbx_version(void);

/* Context::Context / MPIdata::set(1,1,1,1): one process, one GPU. */
int qbx_create(qbx_context** ctx, int device, int precision);
void qbx_destroy(qbx_context* ctx);
const char* qbx_last_error(const qbx_context* ctx);
int qbx_set_precision(qbx_context* ctx, int precision);

/* Basis::resize (src/Basis.cpp:255-643) for the wavefunctions at ecut and
 * the density at 4*ecut, the dense FFT grid of ChargeDensity
 * (src/ChargeDensity.cpp:36-49), and Wavefunction::set_nel / update_occ for
 * nst doubly occupied bands.  xc is "LDA" or "PBE".  cell holds a0,a1,a2. */
int qbx_set_cell(qbx_context* ctx, const double cell[9], double ecut, int nst,
                 const char* xc);
/* Sizes: wavefunction and density basis sizes and the grid. */
int qbx_basis_sizes(const qbx_context* ctx, int* ngw, int* ngv, int np[3]);
/* Miller indices (3*ngw ints) of the wavefunction basis, default order. */
int qbx_basis_miller(const qbx_context* ctx, int* hkl);
/* Use the caller's coefficient order: hkl = 3*ngw Miller indices, one per
 * coefficient row as the caller stores them (NULL restores the default). */
int qbx_set_coeff_order(qbx_context* ctx, const int* hkl);

/* Species::initialize_slpp (src/Species.cpp:510-1055) from the radial
 * tables of a semilocal norm-conserving species: local potential vlocal on
 * a uniform mesh r_i = i*mesh_spacing, nproj projectors proj[iop*nmesh+i]
 * of angular momentum proj_l[iop] (0 or 1) with diagonal D-matrix entries
 * dmat[iop].  Returns the species index in *isp. */
int qbx_add_species(qbx_context* ctx, int zval, double mesh_spacing, int nmesh,
                    const double* vlocal, int nproj, const int* proj_l,
                    const double* proj, const double* dmat, int* isp);

/* EnergyFunctional::atoms_moved (src/EnergyFunctional.cpp:1047-1197) and
 * NonLocalPotential::update_twnl: structure factors, local potential,
 * pseudocharges, E_sr and projectors for positions tau (bohr, 3 per atom,
 * species-major; na[isp] atoms of each species added so far). */
int qbx_set_atoms(qbx_context* ctx, const int* na, const double* tau);

/* SlaterDet coefficients (src/SlaterDet.h:35-109): upload / download.
 * qbx_set_coeffs starts a new stepper history (as a freshly loaded
 * wavefunction does); the _async forms keep it, for callers that keep the
 * SlaterDet in host memory and stream it through every step. */
int qbx_set_coeffs(qbx_context* ctx, const double* c);
int qbx_get_coeffs(qbx_context* ctx, double* c);
/* Upload/download without synchronising the host (pinned buffers). */
int qbx_set_coeffs_async(qbx_context* ctx, const double* c);
int qbx_get_coeffs_async(qbx_context* ctx, double* c);

/* SlaterDet::gram (src/SlaterDet.cpp:480-534). */
int qbx_gram(qbx_context* ctx);

/* ChargeDensity::update_density (src/ChargeDensity.cpp:136-198). */
int qbx_update_density(qbx_context* ctx, double* total_charge);
int qbx_get_density(qbx_context* ctx, double* rhor);

/* EnergyFunctional::update_vhxc (src/EnergyFunctional.cpp:231-394). */
int qbx_update_vhxc(qbx_context* ctx);
int qbx_get_vr(qbx_context* ctx, double* vr);

/* EnergyFunctional::energy(compute_hpsi, dwf, compute_forces, fion, ...)
 * (src/EnergyFunctional.cpp:397-1044) including NonLocalPotential::energy
 * (src/NonLocalPotential.cpp:1258-2069) and SlaterDet::rs_mul_add
 * (src/SlaterDet.cpp:410-477).  fion (3 per atom) may be NULL. */
int qbx_energy(qbx_context* ctx, int compute_hpsi, int compute_forces,
               double* energies, double* fion);
int qbx_get_hpsi(qbx_context* ctx, double* hc);

/* Wavefunction::dot(dwf) (src/SlaterDet.cpp:1122-1153). */
int qbx_eigenvalue_sum(qbx_context* ctx, double* eigsum);

/* PSDAWavefunctionStepper::update (src/PSDAWavefunctionStepper.cpp:46-249),
 * ending with SlaterDet::ortho_align (src/SlaterDet.cpp:768-876). */
int qbx_psda_update(qbx_context* ctx);
int qbx_psda_reset(qbx_context* ctx);

/* WavefunctionStepper choice (the reference's `set wf_dyn`, src/WfDyn.h):
 * "PSDA" (default) or "JD"; qbx_scf_step then ends with that update. */
int qbx_set_wf_dyn(qbx_context* ctx, const char* wf_dyn);
/* JDWavefunctionStepper::update (src/JDWavefunctionStepper.cpp:47-376):
 * after qbx_energy (which leaves H*C), Rayleigh-Ritz on span(C, Z) with the
 * preconditioned residual Z; includes a second H*psi (on Z), whose energy
 * terms the context then holds, as the reference's energy functional does. */
int qbx_jd_update(qbx_context* ctx);

/* Streamed SlaterDet (no counterpart in the reference, whose coefficients
 * stay in host memory): the coefficients live in pinned host memory and
 * pass through the GPU every step.  qbx_stream_in enqueues the upload of a
 * step's input on a copy stream; qbx_scf_step_async enqueues the step (its
 * captured graph, once qbx_set_step_graph has captured it; otherwise the
 * synchronous step) after that upload; qbx_stream_out enqueues the download
 * of the step's result on a second copy stream.  None of them waits for the
 * GPU, so one step's copies overlap its neighbours' compute; the host
 * buffers must stay untouched until qbx_stream_wait, which waits for all of
 * it and returns the last step's energies (and its status as an error). */
int qbx_stream_in(qbx_context* ctx, const double* c_pinned);
int qbx_scf_step_async(qbx_context* ctx);
int qbx_stream_out(qbx_context* ctx, double* c_pinned);
int qbx_stream_wait(qbx_context* ctx, double* energies);

/* k points off Gamma: Wavefunction::add_kpoint for each of nkp k points
 * (kpoints: 3 per k point, units of the reciprocal vectors; weights sum to
 * one) with the Gamma point removed (del_kpoint), src/Wavefunction.cpp:
 * 400-485.  Each k point gets a complex basis {G: |k+G|^2 < 2 ecut}
 * (src/Basis.cpp:449-486) and a complex SlaterDet; qbx_gram,
 * qbx_update_density, qbx_energy (forces and stress excepted),
 * qbx_eigenvalue_sum, qbx_psda_update and qbx_scf_step then work on the k
 * points with the reference's k-weighted sums, in FP64.  nkp = 0 returns
 * to the Gamma point.  Call after qbx_set_cell. */
int qbx_set_kpoints(qbx_context* ctx, int nkp, const double* kpoints,
                    const double* weights);
/* Basis size and Miller indices (3*ngw ints, may be NULL) of k point ikp,
 * in the order of its coefficients (sorted h, k, l). */
int qbx_kpoint_basis(const qbx_context* ctx, int ikp, int* ngw, int* hkl);
/* Coefficients (ngw x nst complex, band-major) and H*psi of k point ikp. */
int qbx_set_kpoint_coeffs(qbx_context* ctx, int ikp, const double* c);
int qbx_get_kpoint_coeffs(qbx_context* ctx, int ikp, double* c);
int qbx_get_kpoint_hpsi(qbx_context* ctx, int ikp, double* hc);

/* One electronic step of the SCF loop with nite = 0
 * (src/BOSampleStepper.cpp:795-977): update_density, update_vhxc,
 * energy(true,...), eigenvalue_sum, PSDA update.  compute_forces: bit 0
 * computes the ionic forces (fion), bit 1 the stress tensor of the step's
 * input state (read it with qbx_get_stress). */
int qbx_scf_step(qbx_context* ctx, int compute_forces, double* energies,
                 double* fion);

/* No counterpart in the reference (one Qbox process runs one sample).  One
 * electronic step of each of n independent contexts (different cells,
 * cutoffs and band counts allowed), run concurrently.  When every context
 * has its step captured as a graph (qbx_set_step_graph), one thread
 * launches every context's graph on that context's stream and then collects
 * the energies (with the environment variable QBX_BATCH_GRAPH=1 at
 * qbx_create of ctxs[0]: the steps are captured together as the branches of
 * one graph cached on ctxs[0], one launch per batch step); otherwise each
 * context is driven by its own host thread.
 * Either way the GPU overlaps the systems.  energies receives
 * n * QBX_NENERGY values (may be NULL); forces are not returned
 * (compute_forces bit 0 only selects the forces variant of the step, bit 1
 * computes each context's stress for qbx_get_stress).  Returns the first
 * failing context's status; its qbx_last_error holds the message.  The
 * contexts must be distinct and not used by other threads meanwhile. */
int qbx_scf_step_batch(qbx_context** ctxs, int n, int compute_forces,
                       double* energies);

/* The <wavefunction> element of a Qbox sample file, as Wavefunction::print
 * writes it with base64 encoding (src/Wavefunction.cpp:919-962,
 * SlaterDet::print src/SlaterDet.cpp:1382-1549): each band's real values on
 * the wavefunction basis's own FFT grid (src/Basis.cpp:509-521), x fastest,
 * base64 in 72-character lines.  The transforms run on the device. */
int qbx_write_wavefunction(qbx_context* ctx, const char* path);
/* Reads such an element (written by this library or by the reference) into
 * the context's coefficients: each grid function transformed forward onto
 * the basis, the diagonal density matrix as the occupations
 * (src/WavefunctionHandler.cpp).  The file's grid must be this basis's
 * grid; only real (Gamma) base64 grid functions. */
int qbx_read_wavefunction(qbx_context* ctx, const char* path);

/* The ground-state SCF loop of BOSampleStepper::step(0) with atoms fixed
 * (src/BOSampleStepper.cpp:781-1114) and wf_dyn = PSDA: nitscf
 * iterations.  With nite > 0 each iteration mixes the new density into the
 * input density (AndersonMixer with mix_ndim history vectors,
 * src/AndersonMixer.cpp, and Kerker weights of radius mix_rcut bohr with
 * coefficient mix_coeff, src/BOSampleStepper.cpp:318-410, 805-881; the
 * reference's charge_mix_ndim, charge_mix_rcut, charge_mix_coeff; mix_ndim 0
 * mixes linearly), rebuilds the potentials and runs up to nite electronic
 * steps, stopping when the eigenvalue sum moves less than 0.01 of the
 * Hartree energy change; with nite = 0 each iteration is one qbx_scf_step
 * without forces.  Stops early when the last three Harris-Foulkes energies
 * lie within scf_tol.  Outputs (each may be NULL): etotal_int[nitscf]
 * (Harris-Foulkes estimate per iteration, :1075-1101),
 * eigsum[nitscf * max(nite,1)] (eigenvalue sum of each electronic step),
 * nite_done[nitscf], nitscf_done (iterations run). */
int qbx_scf_run(qbx_context* ctx, int nitscf, int nite, double mix_coeff,
                double mix_rcut, int mix_ndim, double scf_tol,
                double* etotal_int, double* eigsum, int* nite_done,
                int* nitscf_done);

/* AtomSet::set_positions followed by EnergyFunctional::atoms_moved
 * (src/EnergyFunctional.cpp:1047-1197): the same atoms at new positions
 * tau (species-major, 3 per atom, bohr).  Structure factors, local
 * potential, pseudocharges, projector phases and E_sr are updated in place,
 * so captured steps (qbx_set_step_graph) stay valid. */
int qbx_move_atoms(qbx_context* ctx, const double* tau);

/* BOSampleStepper::step(niter) with atoms_dyn = MD
 * (src/BOSampleStepper.cpp:412-1420): per ionic step the energy and forces
 * at the current positions, MDIonicStepper's velocity Verlet
 * (src/MDIonicStepper.cpp:8-273, no thermostat), qbx_move_atoms, the linear
 * wavefunction extrapolation (first step c + dt v then gram; later steps
 * 2c - c_prev after SlaterDet::align, then SlaterDet::lowdin) and nitscf
 * electronic steps (qbx_scf_step, PSDA); at the end the wavefunction
 * velocity and the forces at the last positions.  The wavefunction
 * velocity persists in the context across calls (the reference's
 * Sample::wfv).  mass_amu: per species (atomic mass units).  vel (may be
 * NULL): initial velocities in, final out (3 per atom, species-major).
 * tau_out (may be NULL): final positions.  ionic (may be NULL): niter x 3
 * values (etotal, ekin_ion, econst = etotal + ekin_ion) of each ionic step.
 * scf (may be NULL): niter * nitscf * QBX_NENERGY energies of the
 * electronic steps. */
int qbx_md_run(qbx_context* ctx, int niter, int nitscf, double dt,
               const double* mass_amu, double* vel, double* tau_out,
               double* ionic, double* scf);

/* DoubleMatrix::polar (src/Matrix.cpp:2446-2540), the orthogonal polar
 * factor used by SlaterDet::ortho_align: x (nst x nst, column-major, host)
 * is replaced by its polar factor.  Bjorck-Bowie steps while
 * ||I - x^T x||_F < 1, Higham steps x <- (x + x^-T)/2 otherwise, stopping
 * after the step in which the norm is <= tol or after maxiter steps.
 * graph != 0 runs the loop as the captured step does (a CUDA graph whose
 * WHILE and IF/ELSE conditional nodes decide on the device).  iters (may be
 * NULL) receives the number of steps. */
int qbx_polar(qbx_context* ctx, double* x, double tol, int maxiter, int graph,
              int* iters);

/* No counterpart in the reference.  on != 0: qbx_scf_step (PSDA, with or
 * without forces; not JD, not stress, not while profiling) runs as a CUDA
 * graph.  Each configuration (first step / later steps with the Anderson
 * extrapolation, with / without forces) runs eagerly once, which sizes every
 * lazily grown buffer, and is captured on its second use; later steps launch
 * the graph.  Inside, the reductions stay in device slots, the Anderson
 * theta is formed on the device and the polar iteration of ortho_align is a
 * conditional WHILE node; the host reads the scalars once after the graph.
 * Changing the cell, precision, GEMM backend, stepper or FFT tuning, or
 * qbx_set_atoms, drops the graphs (qbx_move_atoms keeps them).  A step that cannot be captured turns graphs off and
 * runs eagerly; qbx_step_graph_info then reports why. */
int qbx_set_step_graph(qbx_context* ctx, int on);
/* captured: graphs currently instantiated (0-4); launches: this context's
 * captured steps launched so far (alone or inside a batch graph);
 * batch_launches: batch graphs launched with this context first in the
 * list; note (may be NULL): why capture (or the batch graph) was abandoned,
 * empty if it was not. */
int qbx_step_graph_info(qbx_context* ctx, int* captured, long* launches,
                        long* batch_launches, char* note, int note_len);

/* The stress tensor of EnergyFunctional::energy(..., compute_stress=true,
 * sigma) (src/EnergyFunctional.cpp:440-1044, XCPotential::compute_stress
 * src/XCPotential.cpp:467-640, NonLocalPotential::energy's stress
 * src/NonLocalPotential.cpp:1790-2069, E_sr src/EnergyFunctional.cpp:
 * 1112-1194) for the state of the last qbx_energy call: call it after
 * qbx_energy and before anything that changes C or the potentials.
 * sigma[6] in the order xx yy zz xy yz xz (Hartree/bohr^3); parts (may be
 * NULL) receives 36 values: the ekin, eps, enl, ehart, exc and esr parts,
 * 6 each. */
int qbx_stress(qbx_context* ctx, double* sigma, double* parts);
/* The stress computed by the last qbx_scf_step with bit 1 of
 * compute_forces set (or the last qbx_stress). */
int qbx_get_stress(qbx_context* ctx, double* sigma, double* parts);

/* FourierTransform::backward(c1, c2, f) on the density grid
 * (src/FourierTransform.cpp:193-205): two bands n1, n2 of the current
 * wavefunctions to the complex grid f (2*np012 doubles, host). */
int qbx_ft_backward_pair(qbx_context* ctx, int n1, int n2, double* f);

int qbx_synchronize(qbx_context* ctx);

/* Timer/TimerMap equivalent (src/Timer.h:21-76): CUDA-event timing of the
 * library's named regions on its stream ("xy_vpsi", "gemm_nl_project",
 * "update_density", ...).  qbx_profile(ctx, 1) clears and starts recording;
 * qbx_profile_get returns the total milliseconds and count of one region. */
int qbx_profile(qbx_context* ctx, int on);
int qbx_profile_get(qbx_context* ctx, const char* name, double* ms,
                    long* count);
/* Number of kernels of this library launched on the context so far. */
int qbx_launch_count(qbx_context* ctx, long* n);
/* The cudaStream_t all work of the context is ordered on. */
void* qbx_stream(qbx_context* ctx);
/* Mixed path only: 0 = split BF16 products through cuBLAS, 1 = through the
 * library's tcgen05 kernel (default; shapes it does not cover use cuBLAS). */
int qbx_set_gemm_backend(qbx_context* ctx, int backend);
/* One split-precision product D (m x n) = A^T B of host FP64 matrices A
 * (k x m) and B (k x n), column-major, for checking the products on their
 * own: backend 0 = BF16 splits through cuBLAS, 1 = BF16 splits through the
 * library's tcgen05 kernel, 2 = TF32 splits through the tcgen05 kernel, 3 / 4
 * = BF16 / TF32 splits with A read as an MN-major operand (the form of the
 * tall updates; needs the default 256 x 256 CTA-pair kernel). */
/* No counterpart in the reference (it applies its Cholesky factors with
 * ScaLAPACK triangular solves, src/SlaterDet.cpp:1272-1314).  li = l^-1 for a
 * lower-triangular n x n HOST matrix l (column-major; its upper triangle is
 * not read), through the routine that ortho_align and the polar iteration's
 * Cholesky step of the mixed path use: blocked (32 x 32 diagonal inverses,
 * then FP64 GEMMs doubling the block) for n = 32 x a power of two, *blocked
 * = 1; otherwise one triangular solve of I, *blocked = 0 (blocked may be
 * NULL).  For checking that routine on its own. */
int qbx_lower_inverse(qbx_context* ctx, int n, const double* l, double* li, int* blocked);
int qbx_split_gemm_tn(qbx_context* ctx, int m, int n, int k, const double* a,
                      const double* b, double* d, int backend);

/* ---- The reference's classes on the caller's host arrays.
 * A C++ caller that keeps Qbox's FourierTransform, SlaterDet and
 * NonLocalPotential objects (their headers unchanged) implements their
 * methods with these calls; coefficient arrays are ngw complex values per
 * band, band after band, in the context's coefficient order (the caller's,
 * when qbx_set_coeff_order was given); grids hold np0*np1*np2 values, x
 * fastest (FourierTransform::index, src/FourierTransform.h:167-168). */

/* FourierTransform(const Basis& basis, int np0, int np1, int np2)
 * (src/FourierTransform.h:105-110, src/FourierTransform.cpp:97-114) on any
 * basis: hkl holds the Miller index of each of the ngw coefficients in the
 * caller's order; real_basis != 0 for a Gamma half sphere (each coefficient
 * also stands for -G with the conjugate value).  The basis must fit in the
 * grid as Basis::fits_in_grid requires (src/Basis.cpp:139-144), else error
 * 12.  The transforms run on `device` as full-grid line FFTs; coefficients
 * and grids cross the host link on every call. */
typedef struct qbx_ft qbx_ft;
int qbx_ft_create(qbx_ft** ft, int device, int ngw, const int* hkl, int real_basis, int np0,
                  int np1, int np2);
void qbx_ft_destroy(qbx_ft* ft);
const char* qbx_ft_last_error(qbx_ft* ft);
/* FourierTransform::backward(c, f) (src/FourierTransform.h:112,
 * src/FourierTransform.cpp:159-170): f(r) = sum_G c(G) exp(iG.r) on the
 * grid, -G with the conjugate on a real basis; unscaled. */
int qbx_ft_backward(qbx_ft* ft, const double* c, double* f);
/* FourierTransform::backward(c1, c2, f) (src/FourierTransform.h:117-118,
 * src/FourierTransform.cpp:187-200): f = psi_1 + i psi_2 for two bands of a
 * real basis (src/BasisMapping.cpp:666-700). */
int qbx_ft_backward2(qbx_ft* ft, const double* c1, const double* c2, double* f);
/* FourierTransform::forward(f, c) (src/FourierTransform.h:114,
 * src/FourierTransform.cpp:147-157): c(G) = 1/N sum_r f(r) exp(-iG.r).  The
 * reference overwrites f; here f is left as it was. */
int qbx_ft_forward(qbx_ft* ft, double* f, double* c);
/* FourierTransform::forward(f, c1, c2) (src/FourierTransform.h:120-121,
 * src/FourierTransform.cpp:173-184): the two real functions of f = psi_1 +
 * i psi_2 (src/BasisMapping.cpp:716-750); real basis only. */
int qbx_ft_forward2(qbx_ft* ft, double* f, double* c1, double* c2);

/* SlaterDet::compute_density(ft, weight, rho) (src/SlaterDet.h:66,
 * src/SlaterDet.cpp:225-298) of the context's SlaterDet on the context's
 * grid: rho[i] += weight * sum_n occ_n/Omega |psi_n(r_i)|^2, rho a HOST array
 * of np0*np1*np2 doubles (the staged two-band transforms of the
 * electronic step, in the context's precision). */
int qbx_compute_density(qbx_context* ctx, double weight, double* rho);
/* SlaterDet::rs_mul_add(ft, v, sdp) (src/SlaterDet.h:68,
 * src/SlaterDet.cpp:410-477): sdp.c += FFT_fwd(v(r) FFT_bwd(c)) for every
 * band; v a HOST array of np0*np1*np2 doubles, dc the HOST coefficients of
 * sdp (nst bands), added into. */
int qbx_rs_mul_add(qbx_context* ctx, const double* v, double* dc);
/* NonLocalPotential::energy(compute_hpsi, dsd, compute_forces, fion,
 * compute_stress, sigma_enl) (src/NonLocalPotential.h:65-67,
 * src/NonLocalPotential.cpp:1258-2069) alone: E_nl into *enl; with
 * compute_hpsi the nonlocal H*C added into dc (HOST, nst bands); with
 * compute_forces the nonlocal forces (3 per atom, species-major) written to
 * fion; with compute_stress sigma_enl[6] (xx yy zz xy yz xz). */
int qbx_nonlocal_energy(qbx_context* ctx, int compute_hpsi, double* dc, int compute_forces,
                        double* fion, int compute_stress, double* sigma_enl, double* enl);
/* SlaterDet::ortho_align(const SlaterDet& sd) (src/SlaterDet.h:76,
 * src/SlaterDet.cpp:768-876): orthonormalises the context's C and aligns it
 * with sd, given as HOST coefficients (nst bands).  sd is held in the
 * stepper's last-step buffer, so the PSDA history restarts (as after
 * qbx_set_coeffs). */
int qbx_ortho_align(qbx_context* ctx, const double* c_sd);
/* Wavefunction::diag(dwf, eigvec) (src/Wavefunction.h:115,
 * src/Wavefunction.cpp:834-917) at Gamma: the subspace Hamiltonian
 * h = 2 C^T (H C) - c0 hc0^T from the H*C of the last qbx_energy with
 * compute_hpsi, its nst eigenvalues (ascending) into eig (HOST); with
 * eigvec != 0 the context's C becomes C Z (Z the eigenvectors) and its H*C
 * the previous C, as the reference overwrites dwf; the PSDA history
 * restarts.  FP64 products in both precisions. */
int qbx_diag(qbx_context* ctx, int eigvec, double* eig);
/* SlaterDet::dot(const SlaterDet& sd) (src/SlaterDet.h:77,
 * src/SlaterDet.cpp:1122-1153) at Gamma: tr(C^T C_sd) over the real view,
 * +G and -G once each, *d = 2 sum - sum of the G=0 terms. */
int qbx_dot(qbx_context* ctx, const double* c_sd, double* d);

/* ---- Band pairs of one SlaterDet split over GPUs: the reference's state
 * axis (nstb of MPIdata::set, src/MPIdata.cpp:55-121, the columns of c_ in
 * src/SlaterDet.cpp:84-93) for the FFT work of the step.  Each of nranks
 * processes (one GPU each) builds the same context (cell, species, atoms,
 * coefficients) and calls qbx_set_band_shard with its rank and the group's
 * NCCL unique id, which one rank makes with qbx_nccl_unique_id and the
 * caller passes to the others by its own means.  From then on each GPU
 * transforms a contiguous range of about npairs/nranks band pairs in
 * update_density and in the local part of H*psi; the density is summed over
 * the GPUs (ncclAllReduce, src/ChargeDensity.cpp:166) and the H*psi bands
 * are broadcast from their owners, so every GPU continues the step with the
 * whole of both and computes the same products on the same data.  Every
 * rank must make the same calls in the same order.  Gamma only; exclusive
 * with qbx_set_step_graph.  nranks = 1 with an id runs the collectives on a
 * group of one; nranks = 1 with id = NULL switches sharding off.  libnccl.so.2
 * is loaded at the first call (error 70 if it cannot be). */
#define QBX_NCCL_ID_BYTES 128
int qbx_nccl_unique_id(unsigned char id[QBX_NCCL_ID_BYTES]);
int qbx_set_band_shard(qbx_context* ctx, int rank, int nranks,
                       const unsigned char id[QBX_NCCL_ID_BYTES]);
/* Host-only: the band pairs [first_pair, end_pair) that rank of nranks
 * transforms for nst bands (pair p = bands 2p and 2p+1): contiguous ranges
 * whose sizes differ by one at most. */
int qbx_shard_pairs(int nst, int rank, int nranks, int* first_pair, int* end_pair);

/* Size of the device array behind qbx_density_static: 32 MiB. */
#define QBX_STATIC_SCRATCH_BYTES ((size_t)32 << 20)

/* No counterpart in the reference.  ChargeDensity-style density of nst bands
 * for callers that cannot allocate device memory when they need it (code in
 * a host callback or a plug-in where cudaMalloc is not allowed, or a process
 * whose device memory another framework has already divided up).  d_c is a
 * DEVICE array of nst bands (band-major, 2*ngw doubles each, in the default
 * order of qbx_basis_miller; qbx_set_coeff_order does not apply); d_rho is a
 * DEVICE array of np0*np1*np2 doubles that receives
 * sum_n occ_n/Omega |psi_n(r)|^2 (overwritten).  occ is a HOST array of nst
 * occupations, or NULL for 2 per band.  The z-stick scratch, twiddle and
 * weight tables come from one static device array of QBX_STATIC_SCRATCH_BYTES
 * that every GPU loading the library holds until exit; the call allocates
 * nothing.  Error 62 covers every limit of that array, and the message names
 * which one was hit: (1) an FFT length above 4096; (2) the three twiddle
 * tables and the nst band weights above 1 MiB (about 130 000 bands at the
 * grid lengths used here); (3) one band pair's z-sticks above 31 MiB:
 * np2 * (2*nrods-1) complex values per pair (FP32 in the mixed precision,
 * FP64 otherwise), about 4 M values in FP32.  Every call looks up the
 * array's address in the CUDA context current on the calling thread
 * (cudaGetSymbolAddress, which allocates nothing).  All calls share the
 * array and it keeps the last call's contents; calls that overlap on one
 * GPU race.  Runs on the context's stream and synchronizes that stream
 * before returning. */
int qbx_density_static(qbx_context* ctx, const double* d_c, int nst,
                       const double* occ, double* d_rho);

/* No counterpart in the reference (its FFT plans are fixed at build time).
 * Chooses the staged-FFT launch configuration for this context's grid,
 * basis and precision by timing the candidate plane kernels, CTA shapes,
 * band-pair batches and z-stick blocking on the context's own data (after
 * qbx_set_atoms and qbx_set_coeffs).  A summary of the timings and the
 * choice is written to report (report_len bytes, may be NULL). */
int qbx_autotune(qbx_context* ctx, char* report, int report_len);

/* Host-only setup helpers (no GPU needed), exposing the same host code the
 * context uses.  Basis::resize + ChargeDensity grid: basis sizes, grid and
 * (if hkl != NULL) the 3*ngw Miller indices in the default order. */
int qbx_host_basis(const double cell[9], double ecut, int* ngw, int* ngv,
                   int np[3], int* hkl);
/* Basis::resize of the complex basis at k point k (units of the reciprocal
 * vectors, src/Basis.cpp:449-486): its size, the index of the reference's
 * first local coefficient (rod (0,0) moved to the front) and (if hkl !=
 * NULL) the 3*ngw Miller indices in the library's order (sorted h, k, l). */
int qbx_host_kbasis(const double cell[9], double ecut, const double k[3], int* ngw,
                    int* first, int* hkl);
/* Species::initialize_slpp + Species::dvlocg / vnlg (src/Species.cpp:
 * 1133-1185) evaluated at ng values of |G|: vloc[ng], dvloc[ng],
 * vnl[nproj*ng]. */
int qbx_host_species_eval(int zval, double mesh_spacing, int nmesh,
                          const double* vlocal, int nproj, const int* proj_l,
                          const double* proj, int ng, const double* g,
                          double* vloc, double* dvloc, double* vnl);
/* E_sr and its forces (src/EnergyFunctional.cpp:1112-1192); fion has 3 per
 * atom, species-major. */
int qbx_host_esr(const double cell[9], int nsp, const int* na,
                 const double* zv, const double* tau, double* esr,
                 double* fion);

#ifdef __cplusplus
}
#endif
#endif
