"""GPU checks of the pipeline's phase overlap (cpsd_set_phase_overlap).

The SF-CIS Davidson and the ground state + J^(2)/J^(3) run on two library
worker threads with their own streams, then the excited orders: every
energy must equal the sequential order's bit for bit (same kernels, same
operands, different streams), and an error in either phase must come back
to the caller as an error code with the phase named, not as a hang."""
import numpy as np
import pytest

from cpsd_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,digits", [("c2v_nmo48", 0), ("c2v_nmo48", 5)])
def test_overlap_equals_sequential(name, digits):
    s = synth.make(name)
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    sc, par = api.make_system(s), api.make_params(s, batch_roots=1)
    api.set_mixed(digits, 0.0 if digits else 1.0)
    try:
        out = {}
        for ov in (False, True, True):
            api.set_phase_overlap(ov)
            out.setdefault(ov, []).append(api.pipeline(s, sc, ints, par))
    finally:
        api.set_phase_overlap(True)
        api.set_mixed(0)
    ref = out[False][0]
    for run in out[True]:
        for a, b in zip(run, ref):
            assert len(a) == len(b) and not np.isnan(a).any()
            assert np.array_equal(a, b)


def test_overlap_reports_phase_errors():
    s = synth.make("c2v_nmo48")
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    sc = api.make_system(s)
    bad = api.make_params(s, batch_roots=1)
    bad.davidson_dim = 40  # above the device Davidson's limit of 32: the SF-CIS phase fails
    api.set_phase_overlap(True)
    with pytest.raises(api.CpsdError, match="SF-CIS"):
        api.pipeline(s, sc, ints, bad)
    # the library stays usable after the failed call
    good = api.make_params(s, batch_roots=1)
    om, w2, w3 = api.pipeline(s, sc, ints, good)
    assert len(om) == s.nroots and np.isfinite(w3).all()


def test_overlap_reports_ground_phase_errors():
    """A failure in the ground-state phase (its DIIS solver rejects the
    subspace size) while SF-CIS succeeds beside it."""
    s = synth.make("c2v_nmo48")
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    sc = api.make_system(s)
    bad = api.make_params(s, batch_roots=1)
    bad.diis_dim = 20  # above the device DIIS limit of 16
    api.set_phase_overlap(True)
    with pytest.raises(api.CpsdError, match="ground"):
        api.pipeline(s, sc, ints, bad)
    om, w2, w3 = api.pipeline(s, sc, ints, api.make_params(s, batch_roots=1))
    assert np.isfinite(w3).all()
