"""The no-allocation contraction entry point (cpsd_vv2v_dpd_444_noalloc)
against cpsd_vv2v_dpd_444 through the C-ABI.

Both run the same plan; the no-allocation one always on the FP64 tile
kernel, with the plan tables and split-K partial tiles in the library's
fixed 32 MiB device region.  It is also checked against the CPU oracle
directly, with and without the mixed (digit) mode switched on.  Results
must agree to 1e-12 absolute (FP64, O(1) data) on two calls in a row, the
calls after set-up must leave device memory and the
library's scratch arena untouched, and a contraction needing more than the
region must be rejected without touching V3.  This file is collected last
so that it also runs after every other GPU test in one process."""
import numpy as np
import pytest

from cpsd_b200 import api, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(autouse=True)
def _stream():
    api.use_torch_stream()
    yield


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def cases(s):
    """(V1, V2, V3) index specs: ring, particle-particle ladder (split-K at
    nmo=48 / 4 irreps), hole-hole ladder, and a 4x2 -> 4 term with dummies."""
    o, v = s.popo, s.popv
    s2 = 2 if s.nirrep > 1 else 1
    z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
    return [
        ("aeim", [v, v, o, o], (1, 1), s2, "embj", [v, o, v, o], (1, 1), 1, "abij", [v, v, o, o], (1, 1), s2),
        ("abef", [v, v, v, v], (0, 0), 1, "efij", [v, v, o, o], (0, 0), s2, "abij", [v, v, o, o], (0, 0), s2),
        ("mnij", [o, o, o, o], (0, 0), 1, "abmn", [v, v, o, o], (0, 0), s2, "abij", [v, v, o, o], (0, 0), s2),
        ("ijmb", [o, o, o, v], (0, 1), 1, "am..", [v, o, z, z], (1, 1), s2, "abij", [v, v, o, o], (1, 0), s2),
    ]


def operands(s, case, rng):
    t1, p1, i1, y1, t2, p2, i2, y2, t3, p3, i3, y3 = case
    sym = s.sym
    a = rng.standard_normal(sym.idsymsoc(y1, p1[0], p1[1], i1[0], p1[2], p1[3], i1[1]))
    b = rng.standard_normal(sym.idsymsoc(y2, p2[0], p2[1], i2[0], p2[2], p2[3], i2[1]))
    c = rng.standard_normal(sym.idsymsoc(y3, p3[0], p3[1], i3[0], p3[2], p3[3], i3[1]))
    return (dev(a), (p1, i1, y1), t1), (dev(b), (p2, i2, y2), t2), (c, (p3, i3, y3), t3)


@pytest.mark.parametrize("nmo,nirrep", [(24, 1), (24, 8), (48, 4)])
def test_noalloc_matches_allocating_entry(nmo, nirrep):
    s = synth.System(nmo=nmo, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=nirrep)
    api.init(s.nirrep, s.dirprd)
    rng = np.random.default_rng(nmo + nirrep)
    for case in cases(s):
        (a, da, ta), (b, db, tb), (c, dc, tc) = operands(s, case, rng)
        for f2 in (1.0, 0.0, 0.5):
            ref = dev(c)
            api.vv2v_dpd_444(a, da, ta, b, db, tb, ref, dc, tc, 0.7, f2)
            # two calls in a row, each on a fresh copy of V3
            for call in range(2):
                out = dev(c)
                api.vv2v_dpd_444_noalloc(a, da, ta, b, db, tb, out, dc, tc, 0.7, f2)
                torch.cuda.synchronize()
                np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=0, atol=TOL,
                                           err_msg=f"{ta}*{tb}->{tc} f2={f2} call {call}")


@pytest.mark.parametrize("nirrep", [1, 4])
def test_noalloc_matches_oracle(nirrep):
    """The no-allocation entry point against the CPU oracle directly, on
    two calls in a row; with the mixed (int8-digit) mode switched on it
    still computes in FP64 on the tile kernel."""
    import oracle_ffi as of
    s = synth.System(nmo=48, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=20 + nirrep)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    rng = np.random.default_rng(nirrep)
    try:
        for mixed in (0, 5):
            api.set_mixed(mixed, 0.0)
            for case in cases(s):
                (a, da, ta), (b, db, tb), (c, dc, tc) = operands(s, case, rng)
                ref = c.copy()
                assert of.vv2v_dpd(a.cpu().numpy(), of.desc(*da), ta, b.cpu().numpy(), of.desc(*db), tb, ref,
                                   of.desc(*dc), tc, 0.7, 0.5) == 0
                for call in range(2):
                    out = dev(c)
                    api.vv2v_dpd_444_noalloc(a, da, ta, b, db, tb, out, dc, tc, 0.7, 0.5)
                    torch.cuda.synchronize()
                    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0, atol=TOL,
                                               err_msg=f"{ta}*{tb}->{tc} mixed={mixed} call {call}")
    finally:
        api.set_mixed(0)


def test_noalloc_allocates_nothing():
    s = synth.System(nmo=48, nocc_a=4, nocc_b=2, nirrep=4, seed=11)
    api.init(s.nirrep, s.dirprd)
    rng = np.random.default_rng(3)
    ops = [operands(s, case, rng) for case in cases(s)]
    outs = [dev(c) for (_, _, (c, _, _)) in ops]
    # the first call on this device does the set-up
    (a, da, ta), (b, db, tb), (_, dc, tc) = ops[0]
    api.vv2v_dpd_444_noalloc(a, da, ta, b, db, tb, outs[0], dc, tc, 1.0, 1.0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    hw0 = api.lib().cpsd_workspace_high_water()
    for _ in range(2):
        for ((a, da, ta), (b, db, tb), (_, dc, tc)), out in zip(ops, outs):
            api.vv2v_dpd_444_noalloc(a, da, ta, b, db, tb, out, dc, tc, 0.5, 1.0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert api.lib().cpsd_workspace_high_water() == hw0


def test_noalloc_rejects_oversize():
    # particle-particle ladder with 142 virtual spin orbitals in one irrep:
    # its plan needs about 47 MB of tables and split-K partial tiles
    s = synth.System(nmo=80, nocc_a=10, nocc_b=8, nirrep=1, seed=2, skip_abcd=True)
    api.init(s.nirrep, s.dirprd)
    t1, p1, i1, y1, t2, p2, i2, y2, t3, p3, i3, y3 = cases(s)[1]
    sym = s.sym
    g = torch.Generator(device="cuda").manual_seed(5)
    n1 = sym.idsymsoc(y1, p1[0], p1[1], i1[0], p1[2], p1[3], i1[1])
    n2 = sym.idsymsoc(y2, p2[0], p2[1], i2[0], p2[2], p2[3], i2[1])
    n3 = sym.idsymsoc(y3, p3[0], p3[1], i3[0], p3[2], p3[3], i3[1])
    a = torch.randn(n1, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(n2, dtype=torch.float64, device="cuda", generator=g)
    c = torch.randn(n3, dtype=torch.float64, device="cuda", generator=g)
    keep = c.clone()
    with pytest.raises(api.CpsdError, match="holds at most"):
        api.vv2v_dpd_444_noalloc(a, (p1, i1, y1), t1, b, (p2, i2, y2), t2, c, (p3, i3, y3), t3, 0.7, 0.5)
    torch.cuda.synchronize()
    assert torch.equal(c, keep)
