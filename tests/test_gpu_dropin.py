"""The reference itself on this repository's FourierTransform.

oracle/_ref/ref_driver_gpuft is the reference's own single-task build
(oracle/Makefile) with src/FourierTransform.cpp replaced by
qbox-public_b200/qbox_shim/FourierTransform.cpp, which implements the class
behind its unchanged header on the qbx_ft_* entry points of libqbx.  Every
transform of the reference's unchanged electronic-step code - the band
pairs of ChargeDensity::update_density and SlaterDet::rs_mul_add, the
density-basis transforms of update_vhxc, the PBE gradients - then runs on
the GPU.  Its energies and forces must equal those of the reference's own
CPU run (tests/golden) to 1e-8 Ha and 1e-6 Ha/bohr, as the FP64 path's do.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden
from qbx import systems
from oracle import inputs

pytestmark = pytest.mark.gpu

TERMS = ("ekin", "eps", "enl", "ehart", "exc", "esr", "eself", "etotal", "eigenvalue_sum")


@pytest.mark.parametrize("name,nsteps", [("si8", 5), ("si64", 3)])
def test_reference_runs_on_the_gpu_fourier_transform(name, nsteps):
    if not os.path.exists(inputs.GPU_FT_DRIVER):
        pytest.fail("oracle/_ref/ref_driver_gpuft is not built (make -C oracle gpu_ft)")
    g = golden(name)
    with tempfile.TemporaryDirectory() as td:
        out = inputs.run_reference(systems.get(name), td, nsteps, dump_steps=1, forces=True,
                                   threads=os.cpu_count(), driver=inputs.GPU_FT_DRIVER)
    e = out["energies"]
    for it in range(nsteps):
        for k in TERMS:
            ref = g["e_" + k][it]
            assert abs(e[k][it] - ref) < 1e-8 * max(1, abs(ref)), (it, k, e[k][it], ref)
    np.testing.assert_allclose(out["fion0"], g["fion_first"], atol=1e-6)
