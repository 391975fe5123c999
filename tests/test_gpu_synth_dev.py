"""The device build of the synthetic integrals (csrc/synth_dev.cu) equals the
host build (csrc/synth.c) up to the summation order of the (pq|rs) dot
products.  Input preparation for the workloads too large to build on the
host (the batching draw, nmo up to 240 without symmetry)."""
import numpy as np
import pytest

from cpsd_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nirrep", [1, 2, 4, 8])
def test_device_integrals_equal_host_build(nirrep):
    s = synth.System(nmo=18 if nirrep < 8 else 26, nocc_a=5, nocc_b=3, nirrep=nirrep, seed=9)
    t = synth.device_integrals(s)
    for k, v in s.ints.items():
        d = t[k].cpu().numpy()
        assert d.shape == v.shape
        assert np.abs(d - v).max() <= 1e-14 * max(1.0, np.abs(v).max()), k
    assert np.array_equal(t["eorb"].cpu().numpy(), s.eorb)
