"""The Qbox-side replacement bodies (qbox-public_b200/qbox_shim) compile
against the reference's unchanged headers: FourierTransform.h, SlaterDet.h,
NonLocalPotential.h, ChargeDensity.h, EnergyFunctional.h and
PSDAWavefunctionStepper.h.  A member function defined with a signature its
header does not declare fails to compile, so this pins every replaced
signature (src/FourierTransform.h:105-121, src/SlaterDet.h:66-77,
src/NonLocalPotential.h:65-67, src/ChargeDensity.h:58,
src/EnergyFunctional.h:82-84,111, src/PSDAWavefunctionStepper.h:38).
Needs the reference sources (QBOX_REFERENCE_SRC); the one-task MPI header
of oracle/shim stands in for MPI."""
import glob
import os
import subprocess

import pytest

from conftest import ROOT

REF = os.environ.get("QBOX_REFERENCE_SRC", os.path.join(os.path.dirname(ROOT), "reference", "src"))
SHIM = os.path.join(ROOT, "qbox-public_b200", "qbox_shim")


@pytest.mark.parametrize("src", sorted(glob.glob(os.path.join(SHIM, "*.cpp"))),
                         ids=lambda p: os.path.basename(p))
def test_shim_compiles_against_reference_headers(src, tmp_path):
    if not os.path.isfile(os.path.join(REF, "FourierTransform.h")):
        pytest.skip("reference sources not present")
    cmd = ["g++", "-std=c++17", "-c", "-O0", "-Werror=return-type", "-DFFT_NOLIB", "-DADD_",
           "-I" + os.path.join(ROOT, "oracle", "shim"), "-I" + REF,
           "-I" + os.path.join(ROOT, "include"), "-I" + SHIM,
           "-include", os.path.join(ROOT, "oracle", "shim", "pblas_decl.h"),
           src, "-o", str(tmp_path / "out.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_every_replaced_method_has_a_body():
    text = "".join(open(p).read() for p in glob.glob(os.path.join(SHIM, "*.cpp")))
    for sig in ("FourierTransform::FourierTransform(", "FourierTransform::backward(",
                "FourierTransform::forward(", "SlaterDet::compute_density(",
                "SlaterDet::rs_mul_add(", "SlaterDet::ortho_align(", "SlaterDet::dot(",
                "SlaterDet::gram(", "NonLocalPotential::energy(",
                "ChargeDensity::update_density(", "EnergyFunctional::energy(",
                "EnergyFunctional::update_vhxc(", "PSDAWavefunctionStepper::update("):
        assert sig in text, sig
