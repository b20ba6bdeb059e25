"""Band-pair sharding on one GPU: the NCCL path run as a group of one.

With an NCCL id and nranks = 1 the context takes every band pair and still
runs the collectives of a sharded step (the density allreduce and the
broadcast of its H*psi block) on a one-rank communicator.  Its steps must
equal those of an unsharded context (1e-12 Ha; the collectives of one rank
copy nothing), in FP64 and in the mixed precision.  Captured steps are
refused while sharded.  Several GPUs are not available here; the partition
and reduction bookkeeping of several ranks is tested on the CPU
(tests/test_sharding.py)."""
import numpy as np
import pytest

from qbx import capi, systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,precision", [("si8", capi.FP64), ("si64", capi.MIXED)])
def test_group_of_one_equals_unsharded(name, precision):
    s = systems.get(name)
    a = capi.from_system(s, precision=precision)
    b = capi.from_system(s, precision=precision)
    b.set_band_shard(0, 1, capi.nccl_unique_id())
    for _ in range(3):
        ra = a.scf_step(forces=True)
        rb = b.scf_step(forces=True)
        assert abs(ra["etotal"] - rb["etotal"]) < 1e-12 * max(1.0, abs(ra["etotal"]))
        np.testing.assert_allclose(rb["fion"], ra["fion"], atol=1e-12)
    np.testing.assert_allclose(b.density(), a.density(), rtol=0, atol=1e-14)
    with pytest.raises(capi.QbxError):
        b.set_step_graph(True)
    b.set_band_shard(0, 1, None)          # sharding off
    b.set_step_graph(True)
    a.close()
    b.close()
