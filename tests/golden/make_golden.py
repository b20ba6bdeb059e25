"""Generates the golden fixtures in tests/golden/ by running the reference Qbox
electronic step, compiled single-task by oracle/Makefile (oracle/_ref).

    make -C oracle && python tests/golden/make_golden.py

Each fixture holds, for a seeded synthetic system: every energy term of each
SCF step, the ionic forces and the stress tensor at the first and last step, the grid sizes and
basis size, a fixed sample of the density and local potential on the grid,
H*psi and wavefunction coefficients of a few bands (all G for small bases,
a fixed sample of G otherwise), and per-band norms.
The fixtures pin the numpy oracle (oracle/qbox_np.py) in tests/test_oracle.py.
ref_<name>_jd.npz holds a JD-stepper run, ref_<name>_md.npz a molecular
dynamics run and ref_<name>_gs.npz a ground-state SCF run with charge mixing
of the reference's BOSampleStepper; ref_<name>_wf.npz the <wavefunction>
element the reference's Wavefunction::print writes (base64) for a band
sample, with the coefficients it wrote; ref_<name>.npz of a k-point system
(KPOINT_CASES) the PSDA run on its complex bases, with H*psi and the final
coefficients of a few bands of each k point.  ref_si512_b32.npz is a 32-band
sample of the 512-atom cell (its 140^3 grid and 2048 projectors),
ref_si64_30.npz a 30-step PSDA run of the 64-atom PBE cell and
ref_batch4.npz four systems of the 32-system batch; ref_si64_diag.npz the
subspace diagonalisation (Wavefunction::diag) after three PSDA steps.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "qbox-public_b200"))
sys.path.insert(0, ROOT)

from qbx import systems            # noqa: E402
from oracle import inputs          # noqa: E402

CASES = {"si8": 20, "si64": 3, "h2o32": 2}
NSAMPLE = 2048
NBANDS_FULL = 4


def make(name: str, nsteps: int, workdir: str, s=None, stress: bool = True) -> str:
    if s is None:
        s = systems.get(name)
    out = inputs.run_reference(s, workdir, nsteps, dump_steps=1, forces=True,
                               stress=stress, threads=os.cpu_count())
    meta = out["meta"]
    e = out["energies"]
    rng = np.random.default_rng(12345)
    N = meta["np0v"] * meta["np1v"] * meta["np2v"]
    idx = np.sort(rng.choice(N, NSAMPLE, replace=False))
    st = out["step0"]
    ngw = meta["ngw"]
    gidx = np.arange(ngw) if ngw <= 2000 else np.sort(
        rng.choice(ngw, 512, replace=False))
    fx = dict(
        grid=np.array([meta["np0v"], meta["np1v"], meta["np2v"]]),
        ngw=meta["ngw"], nst=meta["nst"], ng_v=meta["ng_v"],
        omega=meta["omega"], nsteps=nsteps,
        sample_idx=idx,
        rhor_sample=st["rhor"].ravel()[idx],
        vr_sample=st["vr"].ravel()[idx],
        rhor_sum=st["rhor"].sum(), vr_sum=st["vr"].sum(),
        g_idx=gidx,
        hc_bands=st["hc"][:NBANDS_FULL, gidx],
        hc_norm2=(np.abs(st["hc"]) ** 2).sum(1),
        final_c_bands=out["final_c"][:NBANDS_FULL, gidx],
        final_c_norm2=(np.abs(out["final_c"]) ** 2).sum(1),
        fion_first=out["fion0"], fion_last=out[f"fion{nsteps - 1}"],
    )
    if stress:
        fx["sigma_first"] = out["sigma0"]
        fx["sigma_last"] = out[f"sigma{nsteps - 1}"]
    for k in ("ekin", "eps", "enl", "ehart", "ecoul", "exc", "esr", "eself",
              "etotal", "eigenvalue_sum"):
        fx["e_" + k] = e[k]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        f"ref_{name}.npz")
    np.savez_compressed(path, **fx)
    return path


def make_jd(name: str, nsteps: int, workdir: str) -> str:
    """The JD stepper (wf_dyn JD): the eigenvalue sum of each step and the
    energy terms the reference holds after each update, i.e. of the
    correction block Z (src/JDWavefunctionStepper.cpp:203-204)."""
    s = systems.get(name)
    out = inputs.run_reference(s, workdir, nsteps, wf_dyn="JD", threads=os.cpu_count())
    e = out["energies"]
    fx = dict(nsteps=nsteps)
    for k in ("ekin", "eps", "enl", "ehart", "ecoul", "exc", "etotal", "eigenvalue_sum"):
        fx["e_" + k] = e[k]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}_jd.npz")
    np.savez_compressed(path, **fx)
    return path


JD_CASES = {"si8": 6}

# Band samples of a large cell: the 512-atom cell's 140^3 grid, its 2048
# projectors and its plane-wave basis with only a few bands (name: system,
# bands, steps), so that the length-140 kernels are pinned to the reference.
SAMPLE_CASES = {"si512_b32": ("si512", 32, 3)}

# Long PSDA trajectories, energies of every step and the final coefficients
# of a few bands (name: system, steps)
LONG_CASES = {"si64_30": ("si64", 30)}

# Subspace diagonalisation after a few PSDA steps (name: steps)
DIAG_CASES = {"si64": 3}


def make_diag(name: str, workdir: str) -> str:
    """Wavefunction::diag(dwf, true) after the PSDA steps: eigenvalues, and
    the rotated coefficients of a few bands at sampled G."""
    nsteps = DIAG_CASES[name]
    s = systems.get(name)
    out = inputs.run_reference(s, workdir, nsteps, wf_dyn="DIAG", threads=os.cpu_count())
    eig = np.loadtxt(os.path.join(workdir, "diag_eig.txt"))
    fc = out["final_c"]
    gidx = np.sort(np.random.default_rng(12345).choice(fc.shape[1], 512, replace=False))
    fx = dict(nsteps=nsteps, eig=eig, g_idx=gidx, final_c_bands=fc[:, gidx],
              e_etotal=out["energies"]["etotal"])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}_diag.npz")
    np.savez_compressed(path, **fx)
    return path


# Systems of the 32-system batch (their indices) and the steps run for each
BATCH_PICK = (0, 9, 18, 27)
BATCH_STEPS = 2


def make_long(name: str, workdir: str) -> str:
    """Energies of every step of a long PSDA run and the final coefficients
    of a few bands at sampled G."""
    sysname, nsteps = LONG_CASES[name]
    s = systems.get(sysname)
    out = inputs.run_reference(s, workdir, nsteps, threads=os.cpu_count())
    e = out["energies"]
    ngw = out["final_c"].shape[1]
    gidx = np.sort(np.random.default_rng(12345).choice(ngw, 512, replace=False))
    fx = dict(nsteps=nsteps, g_idx=gidx, final_c_bands=out["final_c"][:NBANDS_FULL, gidx],
              final_c_norm2=(np.abs(out["final_c"]) ** 2).sum(1))
    for k in ("ekin", "eps", "enl", "ehart", "ecoul", "exc", "esr", "eself",
              "etotal", "eigenvalue_sum"):
        fx["e_" + k] = e[k]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}.npz")
    np.savez_compressed(path, **fx)
    return path


def make_batch(workdir: str) -> str:
    """A few systems of the 32-system batch (uneven cells, cutoffs and band
    counts, LDA): energies of each of BATCH_STEPS steps and the forces of
    the first step, keyed s<index>_."""
    fx = dict(picked=np.array(BATCH_PICK), nsteps=BATCH_STEPS)
    allsys = systems.batch()
    for i in BATCH_PICK:
        s = allsys[i]
        sub = os.path.join(workdir, f"s{i}")
        out = inputs.run_reference(s, sub, BATCH_STEPS, dump_steps=1, forces=True,
                                   threads=os.cpu_count())
        e = out["energies"]
        for k in ("ekin", "eps", "enl", "ehart", "ecoul", "exc", "esr", "eself",
                  "etotal", "eigenvalue_sum"):
            fx[f"s{i}_e_{k}"] = e[k]
        fx[f"s{i}_fion_first"] = out["fion0"]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_batch4.npz")
    np.savez_compressed(path, **fx)
    return path

# MD: (ionic steps, electronic steps per ionic step, dt in a.u.)
MD_CASES = {"si8": (3, 2, 20.0)}


def make_md(name: str, workdir: str) -> str:
    """Molecular dynamics (atoms_dyn MD) through the reference's own
    BOSampleStepper: the printed energies of each ionic step, the final
    positions and velocities, and the final coefficients of a few bands."""
    niter, nitscf, dt = MD_CASES[name]
    s = systems.get(name)
    out = inputs.run_reference_md(s, workdir, niter, nitscf, dt, threads=os.cpu_count())
    fx = dict(niter=niter, nitscf=nitscf, dt=dt, etotal=out["etotal"], econst=out["econst"],
              ekin_ion=out["ekin_ion"], tau=out["tau"], vel=out["vel"],
              final_c_bands=out["final_c"][:NBANDS_FULL],
              final_c_norm2=(np.abs(out["final_c"]) ** 2).sum(1))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}_md.npz")
    np.savez_compressed(path, **fx)
    return path

# SCF with charge mixing: (nitscf, nite, charge_mix_coeff, charge_mix_rcut,
# charge_mix_ndim)
GS_CASES = {"si8": (10, 4, 0.5, 10.0, 3), "si64": (3, 2, 0.5, 10.0, 3)}


def make_gs(name: str, workdir: str) -> str:
    """The ground-state SCF loop with nite > 0 and Anderson/Kerker charge
    mixing through the reference's own BOSampleStepper: printed
    etotal_int per SCF iteration and eigenvalue sums per electronic step,
    final coefficients of a few bands."""
    nitscf, nite, coeff, rcut, ndim = GS_CASES[name]
    s = systems.get(name)
    out = inputs.run_reference_gs(s, workdir, nitscf, nite, coeff, rcut, ndim,
                                  threads=os.cpu_count())
    ngw = out["final_c"].shape[1]
    gidx = np.arange(ngw) if ngw <= 2000 else np.sort(
        np.random.default_rng(12345).choice(ngw, 512, replace=False))
    fx = dict(nitscf=nitscf, nite=nite, mix_coeff=coeff, mix_rcut=rcut, mix_ndim=ndim,
              etotal_int=out["etotal_int"], eigenvalue_sum=out["eigenvalue_sum"], g_idx=gidx,
              final_c_bands=out["final_c"][:NBANDS_FULL, gidx],
              final_c_norm2=(np.abs(out["final_c"]) ** 2).sum(1))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}_gs.npz")
    np.savez_compressed(path, **fx)
    return path


# wavefunction output of the reference (Wavefunction::print, base64): system,
# band sample
WF_CASES = {"si8": 4}


KPOINT_CASES = {"si8k2": 4, "h2o4k2": 3}


def make_kpoint(name: str, nsteps: int, workdir: str) -> str:
    """PSDA steps of the reference on the k points of a system (complex
    bases): energies of each step, a density sample, H*psi of the first step
    and the final coefficients (a few bands at sampled G) of each k point."""
    s = systems.get(name)
    out = inputs.run_reference(s, workdir, nsteps, dump_steps=1, threads=os.cpu_count())
    meta = out["meta"]
    e = out["energies"]
    rng = np.random.default_rng(54321)
    N = meta["np0v"] * meta["np1v"] * meta["np2v"]
    idx = np.sort(rng.choice(N, NSAMPLE, replace=False))
    st = out["step0"]
    fx = dict(grid=np.array([meta["np0v"], meta["np1v"], meta["np2v"]]), nst=meta["nst"],
              nkp=meta["nkp"], nsteps=nsteps, sample_idx=idx,
              rhor_sample=st["rhor"].ravel()[idx], rhor_sum=st["rhor"].sum())
    for ik in range(meta["nkp"]):
        ngw = meta[f"ngw_k{ik}"]
        gidx = np.sort(rng.choice(ngw, 512, replace=False))
        fx[f"k{ik}_ngw"] = ngw
        fx[f"k{ik}_g_idx"] = gidx
        fx[f"k{ik}_hc_bands"] = st[f"k{ik}_hc"][:NBANDS_FULL, gidx]
        fx[f"k{ik}_hc_norm2"] = (np.abs(st[f"k{ik}_hc"]) ** 2).sum(1)
        fc = out[f"final_k{ik}_c"]
        fx[f"k{ik}_final_c_bands"] = fc[:NBANDS_FULL, gidx]
        fx[f"k{ik}_final_c_norm2"] = (np.abs(fc) ** 2).sum(1)
    for k in ("ekin", "eps", "enl", "ehart", "ecoul", "exc", "esr", "eself",
              "etotal", "eigenvalue_sum"):
        fx["e_" + k] = e[k]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}.npz")
    np.savez_compressed(path, **fx)
    return path


def make_wf(name: str, workdir: str) -> str:
    """The sample-file <wavefunction> element the reference writes for the
    orthonormalised seeded coefficients of a band sample, and those
    coefficients."""
    import subprocess
    s = systems.get(name).band_sample(WF_CASES[name])
    path = inputs.write_system(s, workdir)
    subprocess.run([inputs.REF_DRIVER, path, "1", workdir, "0", "0", "PRINT"], check=True,
                   stdout=subprocess.DEVNULL)
    xml = open(os.path.join(workdir, "wf.xml"), "rb").read()
    c = np.fromfile(os.path.join(workdir, "final_c.bin")).reshape(s.nbands, -1, 2)
    fx = dict(nbands=s.nbands, xml=np.frombuffer(xml, dtype=np.uint8),
              c=c[..., 0] + 1j * c[..., 1])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}_wf.npz")
    np.savez_compressed(out, **fx)
    return out


if __name__ == "__main__":
    import tempfile
    names = sys.argv[1:] or (list(CASES) + [n + "_jd" for n in JD_CASES]
                             + [n + "_md" for n in MD_CASES] + [n + "_gs" for n in GS_CASES]
                             + [n + "_wf" for n in WF_CASES] + list(KPOINT_CASES)
                             + list(SAMPLE_CASES) + list(LONG_CASES) + ["batch4"]
                             + [n + "_diag" for n in DIAG_CASES])
    for n in names:
        with tempfile.TemporaryDirectory() as td:
            if n in SAMPLE_CASES:
                sysname, nb, nsteps = SAMPLE_CASES[n]
                print(make(n, nsteps, td, s=systems.get(sysname).band_sample(nb),
                           stress=False))
            elif n in LONG_CASES:
                print(make_long(n, td))
            elif n == "batch4":
                print(make_batch(td))
            elif n.endswith("_diag"):
                print(make_diag(n[:-5], td))
            elif n in KPOINT_CASES:
                print(make_kpoint(n, KPOINT_CASES[n], td))
            elif n.endswith("_wf"):
                print(make_wf(n[:-3], td))
            elif n.endswith("_gs"):
                print(make_gs(n[:-3], td))
            elif n.endswith("_md"):
                print(make_md(n[:-3], td))
            elif n.endswith("_jd"):
                print(make_jd(n[:-3], JD_CASES[n[:-3]], td))
            else:
                print(make(n, CASES[n], td))
