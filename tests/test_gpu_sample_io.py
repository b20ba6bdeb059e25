"""Sample-file wavefunctions (qbx_write_wavefunction, qbx_read_wavefunction)
against the <wavefunction> element the reference's Wavefunction::print wrote
for the same orthonormalised coefficients (tests/golden/ref_si8_wf.npz).

The text outside the base64 blocks must be identical; the base64 payload
holds each band's real values from a different FFT implementation, so it is
compared after decoding (1e-13 of the largest value) with the same line
layout.  Reading the reference's file must give its coefficients (1e-13).
"""
import base64
import re

import numpy as np
import pytest

from conftest import golden
from qbx import capi, systems

pytestmark = pytest.mark.gpu


def _split(xml: str):
    """(text with the base64 blocks removed, list of decoded arrays, list of
    line counts of each block)"""
    parts = re.split(r'(<grid_function[^>]*>\n)(.*?)(</grid_function>)', xml, flags=re.S)
    text, arrays, lines = [], [], []
    for i in range(0, len(parts), 4):
        text.append(parts[i])
        if i + 3 < len(parts):
            text.append(parts[i + 1] + parts[i + 3])
            body = parts[i + 2]
            lines.append([len(l) for l in body.splitlines()])
            arrays.append(np.frombuffer(base64.b64decode("".join(body.split())), dtype="<f8"))
    return "".join(text), arrays, lines


@pytest.fixture(scope="module")
def ref():
    fx = golden("si8_wf")
    return fx, bytes(fx["xml"]).decode()


def test_write_matches_reference(ref, tmp_path):
    fx, xml_ref = ref
    s = systems.si8().band_sample(int(fx["nbands"]))
    ctx = capi.from_system(s, precision=capi.FP64)
    np.testing.assert_allclose(ctx.get_coeffs(), fx["c"], rtol=0, atol=1e-13)
    path = str(tmp_path / "wf.xml")
    ctx.write_wavefunction(path)
    xml = open(path).read()
    t0, a0, l0 = _split(xml_ref)
    t1, a1, l1 = _split(xml)
    assert t1 == t0
    assert l1 == l0
    assert len(a1) == len(a0) == int(fx["nbands"])
    for x, y in zip(a1, a0):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-13 * np.abs(y).max())
    ctx.close()


def test_read_reference_file(ref, tmp_path):
    fx, xml_ref = ref
    s = systems.si8().band_sample(int(fx["nbands"]))
    ctx = capi.from_system(s, precision=capi.FP64, gram=False)
    ctx.set_coeffs(np.zeros_like(fx["c"]))
    path = tmp_path / "ref_wf.xml"
    path.write_text(xml_ref)
    ctx.read_wavefunction(str(path))
    np.testing.assert_allclose(ctx.get_coeffs(), fx["c"], rtol=0, atol=1e-13)
    ctx.close()


def test_round_trip_si64(tmp_path):
    s = systems.si64()
    a = capi.from_system(s, precision=capi.FP64)
    c0 = a.get_coeffs()
    path = str(tmp_path / "wf64.xml")
    a.write_wavefunction(path)
    b = capi.from_system(s, precision=capi.FP64, gram=False)
    b.set_coeffs(np.zeros_like(c0))
    b.read_wavefunction(path)
    np.testing.assert_allclose(b.get_coeffs(), c0, rtol=0, atol=1e-13 * np.abs(c0).max())
    ea, eb = a.scf_step(), b.scf_step()
    assert abs(ea["etotal"] - eb["etotal"]) < 1e-10
    a.close()
    b.close()
