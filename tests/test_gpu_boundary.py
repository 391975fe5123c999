"""Every exported boundary entry point against the oracle, called through
the C-ABI exactly as a reference-side binding would call it:
vv2v_dpd_424 / 442 / 422 / 222 / 224 (src/libsrint/vv2v_dpd_*.f90) with
their own argument lists, the Fortran-ABI vv2v_dpd_444_ (every argument by
reference, hidden character lengths last) and its error behaviour, and the
pair transforms iexpso / icompso / isymtrso (src/libsrint/iexpso.f90,
icompso.f, isymtrso.f).  FP64: 1e-12 absolute on O(1) data."""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import oracle_ffi as of
from cpsd_b200 import api, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

I64, DBL = ctypes.c_int64, ctypes.c_double
Z = np.array([1, 0, 0, 0, 0, 0, 0, 0])


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def p8(v):
    return (I64 * 8)(*[int(x) for x in v])


@pytest.fixture(autouse=True)
def _stream():
    api.use_torch_stream()
    yield


def system(nirrep):
    s = synth.System(nmo=20, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=3 + nirrep)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    return s


def rand(s, rng, pops, iops, sym):
    n = s.sym.idsymsoc(sym, pops[0], pops[1], iops[0], pops[2], pops[3], iops[1])
    return rng.standard_normal(n)


def oracle(a, da, ta, b, db, tb, c, dc, tc, f1, f2):
    ref = c.copy()
    rc = of.vv2v_dpd(a, of.desc(*da), ta, b, of.desc(*db), tb, ref, of.desc(*dc), tc, f1, f2)
    assert rc == 0
    return ref


def _operand(x, pops, iop, sym, typ, n_index):
    """argument list of one operand in the reference's order"""
    out = [api.dptr(x)]
    if n_index == 4:
        out += [p8(pops[0]), p8(pops[1]), I64(iop[0]), p8(pops[2]), p8(pops[3]), I64(iop[1])]
    else:
        out += [p8(pops[0]), p8(pops[1]), I64(iop[0])]
    return out + [I64(sym), typ.encode()]


# (entry point, index counts, letters, operand populations (o/v), iops, syms)
CASES = [
    ("424", (4, 2, 4), ("aeij", "be", "abij"), ("vvoo", "vv", "vvoo"), ((1, 1), (1, 1), (1, 1))),
    ("424", (4, 2, 4), ("aeij", "be", "abij"), ("vvoo", "vv", "vvoo"), ((1, 0), (1, 1), (1, 0))),
    ("442", (4, 4, 2), ("efmn", "efin", "mi"), ("vvoo", "vvoo", "oo"), ((0, 1), (0, 1), (1, 1))),
    ("442", (4, 4, 2), ("afmn", "efmn", "ae"), ("vvoo", "vvoo", "vv"), ((1, 0), (1, 0), (1, 1))),
    ("422", (4, 2, 2), ("fnai", "fn", "ai"), ("vovo", "vo", "vo"), ((1, 1), (1, 1), (1, 1))),
    ("422", (4, 2, 2), ("mnie", "en", "mi"), ("ooov", "vo", "oo"), ((1, 1), (1, 1), (1, 1))),
    ("222", (2, 2, 2), ("ae", "ei", "ai"), ("vv", "vo", "vo"), ((1, 1), (1, 1), (1, 1))),
    ("222", (2, 2, 2), ("am", "mi", "ai"), ("vo", "oo", "vo"), ((1, 1), (1, 1), (1, 1))),
    ("224", (2, 2, 4), ("ai", "bj", "aibj"), ("vo", "vo", "vovo"), ((1, 1), (1, 1), (1, 1))),
    ("224", (2, 2, 4), ("ij", "ab", "abij"), ("oo", "vv", "vvoo"), ((0, 1), (0, 1), (0, 0))),
]


@pytest.mark.parametrize("nirrep", [1, 4])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_rank_entry_points_match_oracle(case, nirrep):
    kind, ranks, letters, spaces, iops = CASES[case]
    s = system(nirrep)
    rng = np.random.default_rng(case * 10 + nirrep)
    sp = {"o": s.popo, "v": s.popv}
    syms = (2 if nirrep > 1 else 1, 1)
    syms = (syms[0], syms[1], s.sym.dp(syms[0], syms[1]))
    descs, arrays, types = [], [], []
    for r, sps, io, sy, t in zip(ranks, spaces, iops, syms, letters):
        pops = [sp[c] for c in sps] + [Z] * (4 - len(sps))
        if r == 2:
            io = (io[0], 1)
        descs.append((pops, io, sy))
        arrays.append(rand(s, rng, pops, io, sy))
        types.append(t)
    for f2 in (1.0, 0.0, 0.5):
        c0 = arrays[2] if f2 != 0.0 else np.full_like(arrays[2], 999.0)
        pad = [t + "." * (4 - len(t)) for t in types]
        ref = oracle(arrays[0], descs[0], pad[0], arrays[1], descs[1], pad[1], c0, descs[2], pad[2], 0.7, f2)
        out = dev(c0)
        args = []
        for x, (pops, io, sy), t, r in zip((dev(arrays[0]), dev(arrays[1]), out), descs, types, ranks):
            args += _operand(x, pops, io, sy, t, r)
        rc = getattr(api.lib(), f"cpsd_vv2v_dpd_{kind}")(*args, DBL(0.7), DBL(f2))
        api.check(rc, kind)
        np.testing.assert_allclose(host(out), ref, rtol=0, atol=1e-12, err_msg=f"{kind} {letters} f2={f2}")


def _fortran_args(a, da, ta, b, db, tb, c, dc, tc, f1, f2):
    """vv2v_dpd_444_ arguments: everything by reference, then the hidden
    character lengths"""
    keep = []

    def ref(x):
        keep.append(x)
        return ctypes.byref(x)

    args = []
    for x, (pops, io, sy), t in ((a, da, ta), (b, db, tb), (c, dc, tc)):
        args += [api.dptr(x), p8(pops[0]), p8(pops[1]), ref(I64(io[0])), p8(pops[2]), p8(pops[3]),
                 ref(I64(io[1])), ref(I64(sy)), ctypes.c_char_p(t.encode())]
    args += [ref(DBL(f1)), ref(DBL(f2))]
    return args, keep


ENGINE_CASES = [
    ("aeim", "vvoo", (1, 1), "embj", "vovo", (1, 1), "abij", "vvoo", (1, 1)),
    ("abef", "vvvv", (0, 0), "efij", "vvoo", (0, 0), "abij", "vvoo", (0, 0)),
    ("ijmb", "ooov", (0, 1), "am..", "vo..", (1, 1), "abij", "vvoo", (1, 0)),
]


@pytest.mark.parametrize("nirrep", [1, 8])
def test_fortran_binding_matches_oracle(nirrep):
    s = system(nirrep)
    rng = np.random.default_rng(nirrep)
    sp = {"o": s.popo, "v": s.popv, ".": Z}
    s2 = 2 if nirrep > 1 else 1
    for t1, q1, i1, t2, q2, i2, t3, q3, i3 in ENGINE_CASES:
        d1 = ([sp[c] for c in q1], i1, 1)
        d2 = ([sp[c] for c in q2], i2, s2)
        d3 = ([sp[c] for c in q3], i3, s2)
        a, b, c = rand(s, rng, *d1), rand(s, rng, *d2), rand(s, rng, *d3)
        ref = oracle(a, d1, t1, b, d2, t2, c, d3, t3, -0.3, 0.5)
        out = dev(c)
        args, keep = _fortran_args(dev(a), d1, t1, dev(b), d2, t2, out, d3, t3, -0.3, 0.5)
        api.lib().vv2v_dpd_444_(*args, ctypes.c_size_t(4), ctypes.c_size_t(4), ctypes.c_size_t(4))
        np.testing.assert_allclose(host(out), ref, rtol=0, atol=1e-12, err_msg=f"{t1}*{t2}->{t3}")
        # the ierr twin: same result, ierr = 0
        out2 = dev(c)
        args, keep2 = _fortran_args(dev(a), d1, t1, dev(b), d2, t2, out2, d3, t3, -0.3, 0.5)
        ierr = I64(99)
        api.lib().vv2v_dpd_444_ierr_(*args, ctypes.byref(ierr), ctypes.c_size_t(4), ctypes.c_size_t(4),
                                     ctypes.c_size_t(4))
        assert ierr.value == 0
        np.testing.assert_allclose(host(out2), ref, rtol=0, atol=1e-12)


def test_fortran_binding_errors():
    """A failed check: the ierr twin returns the code and leaves V3 alone;
    vv2v_dpd_444_ ends the program with status 1 after printing the
    message, as the reference's STOP does."""
    s = system(4)
    rng = np.random.default_rng(0)
    o, v = s.popo, s.popv
    d1, d2, d3 = ([v, v, o, o], (1, 1), 1), ([v, o, v, o], (1, 1), 1), ([v, v, o, o], (1, 1), 1)
    a, b, c = rand(s, rng, *d1), rand(s, rng, *d2), rand(s, rng, *d3)
    out = dev(c)
    # 'x' appears in one tensor only: an invalid specification
    args, keep = _fortran_args(dev(a), d1, "aexm", dev(b), d2, "embj", out, d3, "abij", 1.0, 1.0)
    ierr = I64(0)
    api.lib().vv2v_dpd_444_ierr_(*args, ctypes.byref(ierr), ctypes.c_size_t(4), ctypes.c_size_t(4),
                                 ctypes.c_size_t(4))
    assert ierr.value < 0
    np.testing.assert_array_equal(host(out), c)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    prog = textwrap.dedent(f"""
        import sys, ctypes
        sys.path.insert(0, {os.path.join(root, 'tests')!r})
        import conftest, numpy as np, torch
        import test_gpu_boundary as tb
        from cpsd_b200 import api
        s = tb.system(4)
        o, v = s.popo, s.popv
        d = ([v, v, o, o], (1, 1), 1)
        x = torch.zeros(s.sym.idsymsoc(1, v, v, 1, o, o, 1), dtype=torch.float64, device="cuda")
        args, keep = tb._fortran_args(x, d, "aexm", x, ([v, o, v, o], (1, 1), 1), "embj", x, d, "abij", 1.0, 1.0)
        api.lib().vv2v_dpd_444_(*args, ctypes.c_size_t(4), ctypes.c_size_t(4), ctypes.c_size_t(4))
        print("returned")
    """)
    r = subprocess.run([sys.executable, "-c", prog], capture_output=True, text=True, timeout=300, cwd=root)
    assert r.returncode == 1, (r.returncode, r.stdout, r.stderr)
    assert "returned" not in r.stdout and "ERROR: vv2v_dpd_444" in r.stderr


@pytest.mark.parametrize("nirrep", [1, 4])
def test_pair_transforms_match_oracle(nirrep):
    """iexpso / icompso / isymtrso on both pairs of (v,v|o,o) and (o,o|o,v)
    tensors, each against the oracle's restatement."""
    s = system(nirrep)
    rng = np.random.default_rng(nirrep)
    o, v = s.popo, s.popv
    L = api.lib()

    def opt(pops, iops, sym, t):
        return api.opt(pops, iops, sym, t)

    for pops, sym in (([v, v, o, o], 1), ([o, o, o, v], 2 if nirrep > 1 else 1), ([v, v, v, o], 1)):
        same = [pops[0] is pops[1], pops[2] is pops[3]]
        # iexpso: packed (iop 0 where the pair's spaces agree) -> full
        iin = (0 if same[0] else 1, 0 if same[1] else 1)
        x = rand(s, rng, pops, iin, sym)
        for e0, e1 in ((1, 0), (0, 1), (1, 1)):
            if (e0 and not same[0]) or (e1 and not same[1]):
                continue
            iout = (1 if e0 else iin[0], 1 if e1 else iin[1])
            ref = np.zeros(s.sym.idsymsoc(sym, pops[0], pops[1], iout[0], pops[2], pops[3], iout[1]))
            assert of.lib().o_iexpso(of.ptr(x), of.ptr(ref), ctypes.byref(of.desc(pops, iin, sym)),
                                     I64(e0), I64(e1)) == 0
            out = torch.zeros(len(ref), dtype=torch.float64, device="cuda")
            api.check(L.cpsd_iexpso(ctypes.byref(opt(pops, iin, sym, dev(x))), ctypes.byref(opt(pops, iout, sym, out)),
                                    I64(e0), I64(e1)), "iexpso")
            np.testing.assert_allclose(host(out), ref, rtol=0, atol=1e-14)
        # icompso: full -> packed on the pairs with equal spaces (c = 1 keeps)
        full = (1, 1)
        y = rand(s, rng, pops, full, sym)
        for c0, c1 in ((0, 1), (1, 0), (0, 0)):
            if (c0 != 1 and not same[0]) or (c1 != 1 and not same[1]):
                continue
            iout = (c0, c1)
            ref = np.zeros(s.sym.idsymsoc(sym, pops[0], pops[1], iout[0], pops[2], pops[3], iout[1]))
            assert of.lib().o_icompso(of.ptr(y), of.ptr(ref), ctypes.byref(of.desc(pops, full, sym)),
                                      I64(c0), I64(c1)) == 0
            out = torch.zeros(len(ref), dtype=torch.float64, device="cuda")
            api.check(L.cpsd_icompso(ctypes.byref(opt(pops, full, sym, dev(y))), ctypes.byref(opt(pops, iout, sym, out)),
                                     I64(c0), I64(c1)), "icompso")
            np.testing.assert_allclose(host(out), ref, rtol=0, atol=1e-14)
        # isymtrso: swap the letters of a pair (the output populations swap)
        for w0, w1 in ((1, 0), (0, 1), (1, 1)):
            opops = [pops[1], pops[0], pops[2], pops[3]] if w0 else list(pops)
            if w1:
                opops[2], opops[3] = opops[3], opops[2]
            ref = np.zeros(s.sym.idsymsoc(sym, opops[0], opops[1], 1, opops[2], opops[3], 1))
            assert of.lib().o_isymtrso(of.ptr(y), of.ptr(ref), ctypes.byref(of.desc(pops, full, sym)),
                                       I64(w0), I64(w1)) == 0
            out = torch.zeros(len(ref), dtype=torch.float64, device="cuda")
            api.check(L.cpsd_isymtrso(ctypes.byref(opt(pops, full, sym, dev(y))), ctypes.byref(opt(opops, full, sym, out)),
                                      I64(w0), I64(w1)), "isymtrso")
            np.testing.assert_allclose(host(out), ref, rtol=0, atol=1e-14)
