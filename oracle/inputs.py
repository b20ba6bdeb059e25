"""Writes seeded synthetic systems in the formats the reference oracle reads,
and runs the compiled reference driver (oracle/_ref/ref_driver).

Test infrastructure, not product: only tests/, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of bench.py use this module.
"""
from __future__ import annotations

import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")


def write_species(sp, path: str) -> None:
    """Plain-text species read by oracle/shim/SpeciesReader.cpp."""
    with open(path, "w") as f:
        f.write(f"symbol {sp.name}\natomic_number {sp.atomic_number}\n")
        f.write(f"mass {sp.mass}\nvalence_charge {sp.zval}\n")
        projs = sp.projectors()
        f.write(f"lmax {max([l for l, _ in projs], default=0)}\n")
        f.write(f"mesh_spacing {sp.mesh_spacing}\n")
        v = sp.local_potential()
        f.write(f"local_potential {v.size}\n")
        f.write("\n".join(f"{x:.17e}" for x in v) + "\n")
        for l, p in projs:
            f.write(f"projector {l} 0 {p.size}\n")
            f.write("\n".join(f"{x:.17e}" for x in p) + "\n")
        for l, d in sp.dmatrix():
            f.write(f"d_ij {l} 0 0 {d:.17e}\n")
        f.write("end\n")


def write_coeffs(path: str, hkl: np.ndarray, c: np.ndarray) -> None:
    nb, ngw = c.shape
    with open(path, "wb") as f:
        np.array([ngw, nb], dtype=np.int32).tofile(f)
        np.ascontiguousarray(hkl, dtype=np.int32).tofile(f)
        out = np.empty((nb, ngw, 2))
        out[..., 0] = c.real
        out[..., 1] = c.imag
        out.tofile(f)


def write_system(sysdef, workdir: str, c: Optional[np.ndarray] = None) -> str:
    """Write system.txt (+ species + coefficients) into workdir."""
    os.makedirs(workdir, exist_ok=True)
    hkl = sysdef.miller()
    if c is None:
        c = sysdef.coefficients(hkl)
    write_coeffs(os.path.join(workdir, "coeffs.bin"), hkl, c)
    lines = ["cell " + " ".join(f"{x:.17e}" for x in sysdef.cell.ravel()),
             f"ecut_ry {sysdef.ecut_ry:.17e}", f"nel {sysdef.nel}",
             f"xc {sysdef.xc}"]
    for sp in sysdef.species:
        p = os.path.join(workdir, f"{sp.name}.sp")
        write_species(sp, p)
        lines.append(f"species {sp.name} {p}")
    count = {}
    for isp, pos in sysdef.atoms:
        name = sysdef.species[isp].name
        count[name] = count.get(name, 0) + 1
        lines.append(f"atom {name}{count[name]} {name} "
                     + " ".join(f"{x:.17e}" for x in pos))
    lines.append(f"coeffs {os.path.join(workdir, 'coeffs.bin')}")
    for ik, (k, w) in enumerate(sysdef.kpoints or []):
        p = os.path.join(workdir, f"coeffs_k{ik}.bin")
        hk = sysdef.kmiller(ik)
        write_coeffs(p, hk, sysdef.kcoefficients(ik, hk))
        lines.append(f"kpoint {k[0]:.17e} {k[1]:.17e} {k[2]:.17e} {w:.17e} {p}")
    path = os.path.join(workdir, "system.txt")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


GPU_FT_DRIVER = os.path.join(HERE, "_ref", "ref_driver_gpuft")


def run_reference(sysdef, workdir: str, nsteps: int, dump_steps: int = 0,
                  forces: bool = False, wf_dyn: str = "PSDA",
                  threads: Optional[int] = None, c=None, stress: bool = False,
                  driver: str = REF_DRIVER) -> Dict:
    """Run the compiled reference on sysdef; returns parsed outputs.  With
    stress=True (implies forces) the stress tensor of the force steps is
    read as out["sigma"][step].  driver=GPU_FT_DRIVER runs the same
    reference build with the GPU FourierTransform of qbox-public_b200/qbox_shim
    in place of its own (make -C oracle gpu_ft)."""
    if not os.path.exists(driver):
        raise FileNotFoundError(f"{driver} not built (make -C oracle)")
    path = write_system(sysdef, workdir, c)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
        env["OPENBLAS_NUM_THREADS"] = str(threads)
    subprocess.run([driver, path, str(nsteps), workdir, str(dump_steps),
                    "2" if stress else ("1" if forces else "0"), wf_dyn], check=True, env=env,
                   stdout=subprocess.DEVNULL)
    return load_outputs(workdir)


def run_reference_md(sysdef, workdir: str, niter: int, nitscf: int, dt: float,
                     threads: Optional[int] = None) -> Dict:
    """The reference's BOSampleStepper::step(niter) with atoms_dyn = MD and
    nitscf PSDA electronic steps per ionic step.  Returns the per-ionic-step
    energies it prints (etotal, econst, ekin_ion; 8 decimals), the final
    positions and velocities (natoms x 3) and coefficients (full precision)."""
    import re
    if not os.path.exists(REF_DRIVER):
        raise FileNotFoundError("oracle/_ref/ref_driver not built (make -C oracle)")
    path = write_system(sysdef, workdir)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
        env["OPENBLAS_NUM_THREADS"] = str(threads)
    subprocess.run([REF_DRIVER, path, str(niter), workdir, "0", "0", "MD", str(nitscf),
                    repr(float(dt))], check=True, env=env, stdout=subprocess.DEVNULL)
    log = open(os.path.join(workdir, "md_log.txt")).read()

    def tag(name):
        return np.array([float(x) for x in re.findall(rf"<{name}>\s*(\S+)\s*</{name}>", log)])
    meta = {}
    with open(os.path.join(workdir, "meta.txt")) as fm:
        for line in fm:
            k, v = line.split()
            meta[k] = int(v)
    a = np.fromfile(os.path.join(workdir, "final_c.bin")).reshape(meta["nst"], meta["ngw"], 2)
    return dict(etotal=tag("etotal"), econst=tag("econst"), ekin_ion=tag("ekin_ion"),
                etotal_int=tag("etotal_int"),
                tau=np.loadtxt(os.path.join(workdir, "md_tau.txt")).reshape(-1, 3),
                vel=np.loadtxt(os.path.join(workdir, "md_vel.txt")).reshape(-1, 3),
                final_c=a[..., 0] + 1j * a[..., 1])


def run_reference_gs(sysdef, workdir: str, nitscf: int, nite: int, mix_coeff: float = 0.5,
                     mix_rcut: float = 10.0, mix_ndim: int = 3,
                     threads: Optional[int] = None) -> Dict:
    """The reference's BOSampleStepper::step(0): nitscf SCF iterations with
    nite PSDA steps each and charge mixing.  Returns the printed etotal_int
    of each iteration and eigenvalue sums of each electronic step
    (8 decimals) and the final coefficients (full precision)."""
    import re
    if not os.path.exists(REF_DRIVER):
        raise FileNotFoundError("oracle/_ref/ref_driver not built (make -C oracle)")
    path = write_system(sysdef, workdir)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
        env["OPENBLAS_NUM_THREADS"] = str(threads)
    subprocess.run([REF_DRIVER, path, str(nitscf), workdir, "0", "0", "GS", str(nite),
                    repr(float(mix_coeff)), repr(float(mix_rcut)), str(int(mix_ndim))],
                   check=True, env=env, stdout=subprocess.DEVNULL)
    log = open(os.path.join(workdir, "gs_log.txt")).read()

    def tag(name):
        return np.array([float(x) for x in re.findall(rf"<{name}>\s*(\S+)\s*</{name}>", log)])
    meta = {}
    with open(os.path.join(workdir, "meta.txt")) as fm:
        for line in fm:
            k, v = line.split()
            meta[k] = int(v)
    a = np.fromfile(os.path.join(workdir, "final_c.bin")).reshape(meta["nst"], meta["ngw"], 2)
    return dict(etotal_int=tag("etotal_int"), eigenvalue_sum=tag("eigenvalue_sum"),
                final_c=a[..., 0] + 1j * a[..., 1])


def load_outputs(workdir: str) -> Dict:
    out: Dict = {}
    meta = {}
    with open(os.path.join(workdir, "meta.txt")) as f:
        for line in f:
            k, v = line.split()
            meta[k] = float(v) if "." in v else int(v)
    out["meta"] = meta
    e = np.loadtxt(os.path.join(workdir, "energies.txt"), ndmin=2)
    names = ["step", "ekin", "econf", "eps", "enl", "ecoul", "exc", "esr",
             "eself", "ehart", "etotal", "eigenvalue_sum", "t_charge",
             "t_vhxc", "t_energy", "t_wf_update"]
    out["energies"] = {n: e[:, i] for i, n in enumerate(names)}
    nst, ngw = meta["nst"], meta["ngw"]
    nkp = meta.get("nkp", 1)
    kfiles = os.path.exists(os.path.join(workdir, "final_k0_c.bin"))
    grid = (meta["np2v"], meta["np1v"], meta["np0v"])
    s = 0
    while os.path.exists(os.path.join(workdir, f"step{s}_rhor.bin")):
        pre = os.path.join(workdir, f"step{s}_")
        d = {}
        d["rhor"] = np.fromfile(pre + "rhor.bin").reshape(grid)
        d["vr"] = np.fromfile(pre + "vr.bin").reshape(grid)
        if kfiles:
            for ik in range(nkp):
                for k in ("hc", "c"):
                    a = np.fromfile(pre + f"k{ik}_{k}.bin").reshape(nst, meta[f"ngw_k{ik}"], 2)
                    d[f"k{ik}_{k}"] = a[..., 0] + 1j * a[..., 1]
        else:
            for k in ("hc", "c"):
                a = np.fromfile(pre + f"{k}.bin").reshape(nst, ngw, 2)
                d[k] = a[..., 0] + 1j * a[..., 1]
        out[f"step{s}"] = d
        s += 1
    for s in range(int(e[-1, 0]) + 1):
        fp = os.path.join(workdir, f"step{s}_fion.txt")
        if os.path.exists(fp):
            out[f"fion{s}"] = np.loadtxt(fp).reshape(-1, 3)
        fs = os.path.join(workdir, f"step{s}_sigma.txt")
        if os.path.exists(fs):
            out[f"sigma{s}"] = np.loadtxt(fs)
    for ik in range(nkp if kfiles else 0):
        a = np.fromfile(os.path.join(workdir, f"final_k{ik}_c.bin")).reshape(
            nst, meta[f"ngw_k{ik}"], 2)
        out[f"final_k{ik}_c"] = a[..., 0] + 1j * a[..., 1]
    fc = os.path.join(workdir, "final_c.bin")
    if os.path.exists(fc):
        a = np.fromfile(fc).reshape(nst, ngw, 2)
        out["final_c"] = a[..., 0] + 1j * a[..., 1]
    return out
