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


def test_concurrent_callers_do_not_starve_the_workers():
    """Three host threads run overlapped pipelines at once (ctypes releases
    the GIL): each pipeline holds two library workers, its ground-state one
    waiting for its SF-CIS one, so the pool must grow with the callers; the
    energies equal the same pipelines run alone."""
    import threading
    names = ["c2v_nmo48", "c2v_nmo48", "c2v_nmo48"]
    mols = [synth.make(n, seed=k) for k, n in enumerate(names)]
    api.init(mols[0].nirrep, mols[0].dirprd)
    api.set_mixed(0)  # the callers' threads start in the library's default (FP64) mode
    ints = [api.DeviceIntegrals(s) for s in mols]
    api.set_phase_overlap(True)
    alone = [api.pipeline(s, api.make_system(s), d, api.make_params(s, batch_roots=1)) for s, d in zip(mols, ints)]
    out, errs = [None] * len(mols), []

    def run(k):
        try:
            s = mols[k]
            out[k] = api.pipeline(s, api.make_system(s), ints[k], api.make_params(s, batch_roots=1))
        except Exception as e:  # reported below
            errs.append(repr(e))

    th = [threading.Thread(target=run, args=(k,), daemon=True) for k in range(len(mols))]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in th), "pipelines did not finish"
    assert not errs, errs
    for a, b in zip(out, alone):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
