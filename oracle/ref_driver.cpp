// Oracle driver: runs the reference Qbox electronic step, single task, on the
// seeded synthetic inputs written by oracle/inputs.py, and dumps energies and
// arrays for the parity tests.  Test infrastructure, not product: it links the
// reference sources compiled by oracle/Makefile into oracle/_ref/.
//
// The loop is the SCF loop of src/BOSampleStepper.cpp:795-977 with nite=0 and
// wf_dyn=PSDA:  ChargeDensity::update_density (:805) -> update_vhxc(false)
// (:891) -> EnergyFunctional::energy(true,...) (:941) -> eigenvalue_sum =
// Wavefunction::dot (:954) -> PSDAWavefunctionStepper::update (:960).
// Input coefficients are keyed by Miller index so the reference's rod order
// (src/Basis.cpp:544-597) never leaks into the inputs.
//
// usage: ref_driver <system.txt> <nsteps> <outdir> [dump_steps=0]
//                   [forces=0] [wf_dyn=PSDA] [nitscf dt]
//        ref_driver <system.txt> <nitscf> <outdir> 0 0 GS <nite> <mix_coeff>
//                   <mix_rcut> <mix_ndim>
// wf_dyn = GS runs the reference's BOSampleStepper::step(0) (ground state,
// atoms fixed) with nitscf SCF iterations of nite PSDA steps each and the
// given charge mixing (charge_mix_coeff, charge_mix_rcut, charge_mix_ndim);
// its log goes to gs_log.txt and the final coefficients to final_c.bin.
// wf_dyn = PRINT writes the orthonormalised input wavefunction with the
// reference's Wavefunction::print (src/Wavefunction.cpp:919-962,
// SlaterDet::print src/SlaterDet.cpp:1382-1549, base64 encoding) to wf.xml
// and its coefficients to final_c.bin.
// wf_dyn = DIAG runs the PSDA steps, then once more update_density,
// update_vhxc and energy(true) and the subspace diagonalisation
// Wavefunction::diag(dwf, true) (src/Wavefunction.cpp:834-917); it writes
// the eigenvalues (diag_eig.txt) and the rotated coefficients (final_c.bin).
// wf_dyn = MD runs the reference's own BOSampleStepper::step(nsteps)
// (src/BOSampleStepper.cpp:165-1428) with atoms_dyn = MD, wf_dyn = PSDA,
// nitscf electronic steps per ionic step, nite = 0 and the time step dt
// (a.u.), no thermostat; its printed output goes to md_log.txt, the final
// positions and velocities to md_tau.txt and md_vel.txt and the final
// coefficients to final_c.bin.
// k points: "kpoint kx ky kz weight coeffs.bin" lines in the system file (k in
// units of the reciprocal vectors) replace the Gamma point by those k points
// (Wavefunction::add_kpoint, del_kpoint; src/Wavefunction.cpp:400-485), each
// with its own complex basis and coefficients keyed by Miller index; the
// PSDA loop then dumps step<N>_k<ik>_{c,hc}.bin and final_k<ik>_c.bin.
// forces = 1: ionic forces at the dumped steps and the last step; forces = 2:
// forces and the stress tensor (EnergyFunctional::energy with
// compute_stress, src/EnergyFunctional.cpp:397-1044), written as
// step<N>_sigma.txt (xx yy zz xy yz xz).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iomanip>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include <sys/time.h>

#include "MPIdata.h"
#include "Sample.h"
#include "Species.h"
#include "SpeciesReader.h"
#include "Atom.h"
#include "Wavefunction.h"
#include "SlaterDet.h"
#include "ChargeDensity.h"
#include "EnergyFunctional.h"
#include "Preconditioner.h"
#include "PSDAWavefunctionStepper.h"
#include "JDWavefunctionStepper.h"
#include "BOSampleStepper.h"
#include "FourierTransform.h"
#include "Basis.h"
#include "Timer.h"

using namespace std;

static double wall(void)
{ struct timeval tv; gettimeofday(&tv, 0); return tv.tv_sec + 1e-6 * tv.tv_usec; }

struct Key { int h, k, l; bool operator<(const Key& o) const
  { return h != o.h ? h < o.h : ( k != o.k ? k < o.k : l < o.l ); } };

static void write_bin(const string& path, const void* p, size_t bytes)
{
  FILE* f = fopen(path.c_str(), "wb");
  if ( !f ) { cerr << "cannot write " << path << endl; exit(1); }
  fwrite(p, 1, bytes, f);
  fclose(f);
}

int main(int argc, char** argv)
{
  if ( argc < 4 )
  {
    cerr << "usage: ref_driver system.txt nsteps outdir [dump_steps] [forces]"
         << endl;
    return 2;
  }
  const string sysfile = argv[1];
  const int nsteps = atoi(argv[2]);
  const string outdir = argv[3];
  const int dump_steps = argc > 4 ? atoi(argv[4]) : 0;
  const int want_forces = argc > 5 ? atoi(argv[5]) : 0;
  const string wf_dyn = argc > 6 ? argv[6] : "PSDA";

  MPIdata::set(1,1,1,1);
  Sample s;
  s.ctrl.xc = "LDA";
  s.ctrl.ecuts = 0.0;
  s.ctrl.ecutprec = 0.0;
  s.ctrl.polarization = "OFF";
  s.ctrl.fermi_temp = 0.0;
  for ( int i = 0; i < 6; i++ ) s.ctrl.ext_stress[i] = 0.0;
  s.ctrl.e_field = D3vector(0,0,0);
  s.ctrl.alpha_PBE0 = 0.25;
  s.ctrl.alpha_RSH = 0.0; s.ctrl.beta_RSH = 0.0; s.ctrl.mu_RSH = 0.0;
  s.ctrl.stress = "OFF";
  s.ctrl.wf_diag = "F";
  // every other control field BOSampleStepper and its steppers read
  s.ctrl.timing = "OFF";
  s.ctrl.wf_dyn = "PSDA";
  s.ctrl.atoms_dyn = "LOCKED";
  s.ctrl.nite = 0;
  s.ctrl.emass = 0.0;
  s.ctrl.tcp = "OFF"; s.ctrl.tcp_rcut = 0.0; s.ctrl.tcp_sigma = 0.0;
  s.ctrl.gms_mix = 0.0;
  s.ctrl.thermostat = "OFF";
  s.ctrl.th_temp = 0.0; s.ctrl.th_time = 0.0; s.ctrl.th_width = 0.0;
  s.ctrl.lock_cm = false;
  s.ctrl.cell_dyn = "LOCKED"; s.ctrl.cell_lock = "OFF"; s.ctrl.cell_mass = 0.0;
  s.ctrl.spin = "OFF"; s.ctrl.delta_spin = 0;
  s.ctrl.dt = 0.0; s.ctrl.iprint = 1; s.ctrl.timeout = 0;
  s.ctrl.charge_mix_coeff = 0.5; s.ctrl.charge_mix_rcut = 10.0; s.ctrl.charge_mix_ndim = 0;
  s.ctrl.blHF[0] = s.ctrl.blHF[1] = s.ctrl.blHF[2] = 1; s.ctrl.btHF = 0.0;
  s.ctrl.scf_tol = 0.0; s.ctrl.force_tol = 0.0; s.ctrl.stress_tol = 0.0;
  s.ctrl.iter_cmd = ""; s.ctrl.iter_cmd_period = 1;

  // ---- system file ----
  ifstream in(sysfile.c_str());
  if ( !in ) { cerr << "cannot open " << sysfile << endl; return 1; }
  string key, coeff_file;
  struct KLine { double k[3], w; string path; };
  vector<KLine> klines;
  double a[9] = {0};
  double ecut_ry = 0.0;
  int nel = 0;
  int atom_count = 0;
  while ( in >> key )
  {
    if ( key == "cell" ) for ( int i = 0; i < 9; i++ ) in >> a[i];
    else if ( key == "ecut_ry" ) in >> ecut_ry;
    else if ( key == "nel" ) in >> nel;
    else if ( key == "xc" ) in >> s.ctrl.xc;
    else if ( key == "species" )
    {
      string name, path; in >> name >> path;
      Species* sp = new Species(name);
      SpeciesReader rdr;
      rdr.uri_to_species(path, *sp);
      s.atoms.addSpecies(sp, name);
    }
    else if ( key == "atom" )
    {
      string name, spname; double x, y, z;
      in >> name >> spname >> x >> y >> z;
      s.atoms.addAtom(new Atom(name, spname, D3vector(x,y,z), D3vector(0,0,0)));
      atom_count++;
    }
    else if ( key == "coeffs" ) in >> coeff_file;
    else if ( key == "kpoint" )
    {
      KLine kl; in >> kl.k[0] >> kl.k[1] >> kl.k[2] >> kl.w >> kl.path;
      klines.push_back(kl);
    }
    else { cerr << "unknown key " << key << endl; return 1; }
  }
  UnitCell cell(D3vector(a[0],a[1],a[2]), D3vector(a[3],a[4],a[5]),
                D3vector(a[6],a[7],a[8]));
  s.atoms.set_cell(cell);
  s.wf.resize(cell, cell, 0.5 * ecut_ry);
  s.wf.set_nel(nel);
  s.wf.update_occ(0.0);
  if ( !klines.empty() )
  {
    for ( size_t i = 0; i < klines.size(); i++ )
      s.wf.add_kpoint(D3vector(klines[i].k[0],klines[i].k[1],klines[i].k[2]),
                      klines[i].w);
    s.wf.del_kpoint(D3vector(0,0,0));
  }
  const int nkp = s.wf.nkp();

  // ---- coefficients of each k point, keyed by Miller index ----
  // perms[ikp][ig] = input row of reference coefficient ig
  vector<vector<int> > perms(nkp);
  for ( int ikp = 0; ikp < nkp; ikp++ )
  {
    const string path = klines.empty() ? coeff_file : klines[ikp].path;
    SlaterDet& sdk = *s.wf.sd(0,ikp);
    const Basis& bk = sdk.basis();
    const int ngwk = bk.localsize();
    const int nstk = sdk.nst();
    ComplexMatrix& ck = sdk.c();
    FILE* fc = fopen(path.c_str(), "rb");
    if ( !fc ) { cerr << "cannot open " << path << endl; return 1; }
    int hdr[2];
    if ( fread(hdr, sizeof(int), 2, fc) != 2 ) return 1;
    if ( hdr[0] != ngwk || hdr[1] != nstk )
    {
      cerr << "basis mismatch: file ngw=" << hdr[0] << " nb=" << hdr[1]
           << " reference ngw=" << ngwk << " nst=" << nstk << endl;
      return 1;
    }
    vector<int> hkl(3*ngwk);
    if ( fread(&hkl[0], sizeof(int), 3*ngwk, fc) != (size_t)(3*ngwk) ) return 1;
    vector<double> cin(2*(size_t)ngwk*nstk);
    if ( fread(&cin[0], sizeof(double), cin.size(), fc) != cin.size() ) return 1;
    fclose(fc);
    map<Key,int> row_of;
    for ( int i = 0; i < ngwk; i++ )
      row_of[Key{hkl[3*i],hkl[3*i+1],hkl[3*i+2]}] = i;
    vector<int>& pk = perms[ikp];
    pk.resize(ngwk);
    for ( int ig = 0; ig < ngwk; ig++ )
    {
      Key k{bk.idx(3*ig), bk.idx(3*ig+1), bk.idx(3*ig+2)};
      map<Key,int>::iterator it = row_of.find(k);
      if ( it == row_of.end() ) { cerr << "Miller index missing" << endl; return 1; }
      pk[ig] = it->second;
    }
    for ( int n = 0; n < nstk; n++ )
      for ( int ig = 0; ig < ngwk; ig++ )
      {
        const size_t src = 2*((size_t)n*ngwk + pk[ig]);
        ck[ig + (size_t)n*ck.mloc()] = complex<double>(cin[src], cin[src+1]);
      }
  }
  s.wf.gram();

  SlaterDet& sd = *s.wf.sd(0,0);
  const Basis& basis = sd.basis();
  const int ngw = basis.localsize();
  const int nst = sd.nst();
  ComplexMatrix& c = sd.c();
  const int mloc = c.mloc();
  const vector<int>& perm = perms[0];
  // coefficients of k point ikp of a wavefunction in the input order
  auto input_order = [&](const Wavefunction& w, int ikp) {
    const ComplexMatrix& m = w.sd(0,ikp)->c();
    const vector<int>& pk = perms[ikp];
    const int ngwk = (int)pk.size();
    vector<double> out(2*(size_t)ngwk*nst);
    for ( int n = 0; n < nst; n++ )
      for ( int ig = 0; ig < ngwk; ig++ )
      {
        const complex<double> v = m[ig + (size_t)n*m.mloc()];
        const size_t dst = 2*((size_t)n*ngwk + pk[ig]);
        out[dst] = v.real(); out[dst+1] = v.imag();
      }
    return out;
  };

  if ( wf_dyn == "PRINT" )
  {
    ofstream wo((outdir + "/wf.xml").c_str());
    s.wf.print(wo, "base64", "wavefunction");
    wo.close();
    vector<double> out(2*(size_t)ngw*nst);
    for ( int n = 0; n < nst; n++ )
      for ( int ig = 0; ig < ngw; ig++ )
      {
        const complex<double> v = c[ig + (size_t)n*mloc];
        const size_t dst = 2*((size_t)n*ngw + perm[ig]);
        out[dst] = v.real(); out[dst+1] = v.imag();
      }
    write_bin(outdir + "/final_c.bin", &out[0], out.size()*sizeof(double));
    return 0;
  }

  if ( wf_dyn == "GS" )
  {
    const int nite = argc > 7 ? atoi(argv[7]) : 0;
    s.ctrl.charge_mix_coeff = argc > 8 ? atof(argv[8]) : 0.5;
    s.ctrl.charge_mix_rcut = argc > 9 ? atof(argv[9]) : 10.0;
    s.ctrl.charge_mix_ndim = argc > 10 ? atoi(argv[10]) : 3;
    ofstream log((outdir + "/gs_log.txt").c_str());
    streambuf* saved = cout.rdbuf(log.rdbuf());
    {
      BOSampleStepper stepper(s, nsteps, nite);
      stepper.step(0);
    }
    cout.rdbuf(saved);
    vector<double> out(2*(size_t)ngw*nst);
    for ( int n = 0; n < nst; n++ )
      for ( int ig = 0; ig < ngw; ig++ )
      {
        const complex<double> v = c[ig + (size_t)n*mloc];
        const size_t dst = 2*((size_t)n*ngw + perm[ig]);
        out[dst] = v.real(); out[dst+1] = v.imag();
      }
    write_bin(outdir + "/final_c.bin", &out[0], out.size()*sizeof(double));
    ofstream meta((outdir + "/meta.txt").c_str());
    meta << "ngw " << ngw << "\nnst " << nst << "\nnatoms " << atom_count << "\n";
    return 0;
  }

  if ( wf_dyn == "MD" )
  {
    const int nitscf = argc > 7 ? atoi(argv[7]) : 1;
    s.ctrl.atoms_dyn = "MD";
    s.ctrl.dt = argc > 8 ? atof(argv[8]) : 20.0;
    ofstream log((outdir + "/md_log.txt").c_str());
    streambuf* saved = cout.rdbuf(log.rdbuf());
    {
      BOSampleStepper stepper(s, nitscf, 0);
      stepper.step(nsteps);
    }
    cout.rdbuf(saved);
    vector<vector<double> > tau;
    s.atoms.get_positions(tau);
    ofstream to((outdir + "/md_tau.txt").c_str());
    to << setprecision(17);
    for ( size_t is = 0; is < tau.size(); is++ )
      for ( size_t i = 0; i < tau[is].size(); i++ ) to << tau[is][i] << "\n";
    // MDIonicStepper::compute_v stores the velocities in the AtomSet
    vector<vector<double> > vel;
    s.atoms.get_velocities(vel);
    ofstream vo((outdir + "/md_vel.txt").c_str());
    vo << setprecision(17);
    for ( size_t is = 0; is < vel.size(); is++ )
      for ( size_t i = 0; i < vel[is].size(); i++ ) vo << vel[is][i] << "\n";
    vector<double> out(2*(size_t)ngw*nst);
    for ( int n = 0; n < nst; n++ )
      for ( int ig = 0; ig < ngw; ig++ )
      {
        const complex<double> v = c[ig + (size_t)n*mloc];
        const size_t dst = 2*((size_t)n*ngw + perm[ig]);
        out[dst] = v.real(); out[dst+1] = v.imag();
      }
    write_bin(outdir + "/final_c.bin", &out[0], out.size()*sizeof(double));
    ofstream meta((outdir + "/meta.txt").c_str());
    meta << "ngw " << ngw << "\nnst " << nst << "\nnatoms " << atom_count << "\n";
    return 0;
  }

  // ---- set up the energy functional and the stepper ----
  ChargeDensity cd(s.wf);
  EnergyFunctional ef(s, cd);
  Preconditioner prec(s.wf, ef, s.ctrl.ecutprec);
  TimerMap tmap;
  WavefunctionStepper* stepper = 0;
  if ( wf_dyn == "JD" )
    stepper = new JDWavefunctionStepper(s.wf, prec, ef, tmap);
  else
    stepper = new PSDAWavefunctionStepper(s.wf, prec, tmap);
  Wavefunction dwf(s.wf);
  vector<vector<double> > fion;
  valarray<double> sigma(6);
  fion.resize(s.atoms.nsp());
  for ( int is = 0; is < s.atoms.nsp(); is++ )
    fion[is].resize(3*s.atoms.na(is));

  const FourierTransform& vft = *cd.vft();
  const int np012 = vft.np012();

  ofstream eo((outdir + "/energies.txt").c_str());
  eo << setprecision(17);
  eo << "# step ekin econf eps enl ecoul exc esr eself ehart etotal "
        "eigenvalue_sum t_charge t_vhxc t_energy t_wf_update\n";
  {
    ofstream meta((outdir + "/meta.txt").c_str());
    meta << "ngw " << ngw << "\nnst " << nst << "\nnp0v " << vft.np0()
         << "\nnp1v " << vft.np1() << "\nnp2v " << vft.np2()
         << "\nng_v " << cd.vbasis()->localsize()
         << "\nnrods " << basis.nrods() << "\nomega " << cell.volume()
         << "\nnatoms " << atom_count << "\nnkp " << nkp << "\n";
    for ( int ikp = 0; ikp < nkp; ikp++ )
      meta << "ngw_k" << ikp << " " << perms[ikp].size() << "\n";
  }

  stepper->preprocess();
  for ( int itscf = 0; itscf < nsteps; itscf++ )
  {
    const double t0 = wall();
    cd.update_density();
    const double t1 = wall();
    const bool last = ( itscf == nsteps - 1 );
    const bool fstep = want_forces && ( last || itscf < dump_steps );
    const bool sstep = fstep && want_forces == 2;
    ef.update_vhxc(sstep);
    const double t2 = wall();
    ef.energy(true, dwf, fstep, fion, sstep, sigma);
    const double t3 = wall();
    const double eigsum = real(s.wf.dot(dwf));
    if ( itscf < dump_steps )
    {
      ostringstream pre; pre << outdir << "/step" << itscf << "_";
      write_bin(pre.str() + "rhor.bin", &cd.rhor[0][0], np012 * sizeof(double));
      write_bin(pre.str() + "vr.bin", &ef.v_r[0][0], np012 * sizeof(double));
      // C and H*C in the input (sorted Miller) order
      for ( int ikp = 0; ikp < nkp; ikp++ )
      {
        ostringstream kp;
        if ( !klines.empty() ) kp << "k" << ikp << "_";
        vector<double> out = input_order(dwf, ikp);
        write_bin(pre.str() + kp.str() + "hc.bin", &out[0], out.size()*sizeof(double));
        out = input_order(s.wf, ikp);
        write_bin(pre.str() + kp.str() + "c.bin", &out[0], out.size()*sizeof(double));
      }
    }
    if ( sstep )
    {
      ostringstream fn; fn << outdir << "/step" << itscf << "_sigma.txt";
      ofstream so(fn.str().c_str());
      so << setprecision(17);
      for ( int i = 0; i < 6; i++ )
        so << sigma[i] << "\n";
    }
    if ( fstep )
    {
      ostringstream fn; fn << outdir << "/step" << itscf << "_fion.txt";
      ofstream fo(fn.str().c_str());
      fo << setprecision(17);
      for ( int is = 0; is < s.atoms.nsp(); is++ )
        for ( int i = 0; i < 3*s.atoms.na(is); i++ )
          fo << fion[is][i] << "\n";
    }
    stepper->update(dwf);
    const double t4 = wall();
    eo << itscf << " " << ef.ekin() << " " << ef.econf() << " " << ef.eps()
       << " " << ef.enl() << " " << ef.ecoul() << " " << ef.exc() << " "
       << ef.esr() << " " << ef.eself() << " " << ef.ehart() << " "
       << ef.etotal() << " " << eigsum << " " << (t1-t0) << " " << (t2-t1)
       << " " << (t3-t2) << " " << (t4-t3) << "\n";
    eo.flush();
  }
  if ( wf_dyn == "DIAG" )
  {
    cd.update_density();
    ef.update_vhxc(false);
    ef.energy(true, dwf, false, fion, false, sigma);
    s.wf.diag(dwf, true);
    ofstream ev((outdir + "/diag_eig.txt").c_str());
    ev << setprecision(17);
    const vector<double>& eig = s.wf.sd(0,0)->eig();
    for ( size_t n = 0; n < eig.size(); n++ )
      ev << eig[n] << "\n";
  }
  // final wavefunctions
  for ( int ikp = 0; ikp < nkp; ikp++ )
  {
    ostringstream fn;
    fn << outdir << "/final_" << (klines.empty() ? "" : "k") ;
    if ( !klines.empty() ) fn << ikp << "_";
    fn << "c.bin";
    vector<double> out = input_order(s.wf, ikp);
    write_bin(fn.str(), &out[0], out.size()*sizeof(double));
  }
  delete stepper;
  return 0;
}
