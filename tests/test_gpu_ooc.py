"""Out-of-core particle ladder: abcd in host memory (the reference's
vvvv_incore = .false. case, p_c2_r2abcd_h of src/lib_cc/c2_r2abcd.f90)
streamed through two device staging buffers.  Small staging buffers force
many panels per irrep block; pinned and pageable host memory; the results
equal the device-resident run to rounding and the oracle to 1e-9 Eh."""
import ctypes

import numpy as np
import pytest

import oracle_ffi as of
from cpsd_b200 import api, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _panel():
    api.use_torch_stream()
    yield
    api.check(api.lib().cpsd_set_host_panel_bytes(ctypes.c_size_t(1 << 30)), "panel bytes")


@pytest.mark.parametrize("name,pinned,panel", [("c2v_nmo48", True, 65536), ("c2v_nmo48", False, 1 << 20),
                                               ("d2h_small", True, 32768)])
def test_pipeline_with_host_abcd(name, pinned, panel):
    if name == "d2h_small":
        s = synth.System(nmo=40, nocc_a=5, nocc_b=3, nirrep=8, seed=9, roots=3)
    else:
        s = synth.make(name)
    api.init(s.nirrep, s.dirprd)
    dev = api.DeviceIntegrals(s)
    sc, par = api.make_system(s), api.make_params(s)
    ref = api.pipeline(s, sc, dev, par)
    t = dict(dev.t)
    h = torch.from_numpy(s.ints["abcd"].copy())
    t["abcd"] = h.pin_memory() if pinned else h
    host = api.DeviceIntegrals.from_tensors(t)
    api.check(api.lib().cpsd_set_host_panel_bytes(ctypes.c_size_t(panel)), "panel bytes")
    api.launch_count(True)
    got = api.pipeline(s, sc, host, par)
    for a, b in zip(got, ref):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10)
    oom, ow2, ow3 = of.Oracle(s).pipeline()
    np.testing.assert_allclose(got[1], ow2, rtol=0, atol=1e-9)
    np.testing.assert_allclose(got[2], ow3, rtol=0, atol=1e-9)


def test_ground_with_host_abcd():
    s = synth.make("c2v_nmo48")
    api.init(s.nirrep, s.dirprd)
    dev = api.DeviceIntegrals(s)
    sc, par = api.make_system(s), api.make_params(s)
    g0 = api.ground(s, sc, dev, par)
    t = dict(dev.t)
    t["abcd"] = torch.from_numpy(s.ints["abcd"].copy()).pin_memory()
    host = api.DeviceIntegrals.from_tensors(t)
    api.check(api.lib().cpsd_set_host_panel_bytes(ctypes.c_size_t(40000)), "panel bytes")
    g1 = api.ground(s, sc, host, par)
    assert abs(g1["E3"] - g0["E3"]) < 1e-12
    torch.cuda.synchronize()
    np.testing.assert_allclose(g1["T2_2"].cpu().numpy(), g0["T2_2"].cpu().numpy(), rtol=0, atol=1e-13)


def test_host_ladder_is_fp64_in_mixed_mode():
    """c2_r2abcd with a host abcd while every contraction is routed to the
    int8 digits (min_gflop 0): the streamed ladder stays FP64 and equals
    the FP64 device ladder to rounding, where the digit path would differ
    by its digit error"""
    import oracle_ffi as of  # noqa: F811
    s = synth.System(nmo=40, nocc_a=5, nocc_b=3, nirrep=4, seed=4)
    api.init(s.nirrep, s.dirprd)
    o, v = s.popo, s.popv
    rng = np.random.default_rng(0)
    l2 = s.sym.idsymsoc(1, v, v, 0, o, o, 0)
    r2 = torch.from_numpy(rng.standard_normal(l2)).cuda()
    Vd = torch.from_numpy(s.ints["abcd"]).cuda()
    Vh = torch.from_numpy(s.ints["abcd"].copy()).pin_memory()
    dvv = ([v, v, o, o], (0, 0), 1)
    outs = {}
    for mode in ("fp64", "host_mixed", "dev_mixed"):
        out = torch.zeros(l2, dtype=torch.float64, device="cuda")
        api.set_mixed(0 if mode == "fp64" else 5, 0.0)
        try:
            Vopt = api.opt([v, v, v, v], (0, 0), 1, Vd)
            if mode == "host_mixed":
                Vopt.arr = Vh.data_ptr()
            api.check(api.lib().cpsd_c2_r2abcd(ctypes.byref(api.opt(*dvv, out)), ctypes.byref(api.opt(*dvv, r2)),
                                               ctypes.byref(Vopt), ctypes.c_double(1.0)), "c2_r2abcd")
        finally:
            api.set_mixed(0)
        torch.cuda.synchronize()
        outs[mode] = out.cpu().numpy()
    np.testing.assert_allclose(outs["host_mixed"], outs["fp64"], rtol=0, atol=1e-13)
    assert np.max(np.abs(outs["dev_mixed"] - outs["fp64"])) > 1e-13
