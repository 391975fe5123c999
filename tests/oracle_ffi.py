"""ctypes binding to the CPU oracle (oracle/_build/libcpsd_oracle.so).

Test infrastructure only: used by tests/ and by bench.py's CPU baseline.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libcpsd_oracle.so")
I64 = ctypes.c_int64
DP = ctypes.POINTER(ctypes.c_double)


class ODesc(ctypes.Structure):
    _fields_ = [("pop", (I64 * 8) * 4), ("iop", I64 * 2), ("sym", I64)]


class OOpt(ctypes.Structure):
    _fields_ = [("d", ODesc), ("arr", ctypes.c_void_p), ("len", I64)]


class OSystem(ctypes.Structure):
    _fields_ = [("nirrep", I64), ("dirprd", I64 * 64), ("symry", I64),
                ("popa", I64 * 8), ("popb", I64 * 8), ("vrta", I64 * 8), ("vrtb", I64 * 8),
                ("popo", I64 * 8), ("popv", I64 * 8)]


class OIntegrals(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb")]


class OParams(ctypes.Structure):
    _fields_ = [("davidson_dim", I64), ("davidson_cyc", I64), ("davidson_conv", I64), ("lowest", I64),
                ("diis_dim", I64), ("diis_cyc", I64), ("diis_max_err", ctypes.c_double),
                ("spin_flip", I64), ("open_shell", I64), ("ex_mult", I64),
                ("estate_sym", I64 * 8), ("nthreads", I64)]


class OJints(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("J2_Foo", "J2_Fvv", "J2_Wovvo", "J2_Wovoo",
                                               "J3_Foo", "J3_Fvv", "J3_Wovvo")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle not built: {ORACLE_SO}")
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.o_vv2v_dpd.restype = ctypes.c_int
        _lib.o_ddot = None
    return _lib


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def arr8(v):
    return (I64 * 8)(*[int(x) for x in v])


def set_symmetry(nirrep, dirprd):
    d = np.ascontiguousarray(dirprd, dtype=np.int64)
    rc = lib().o_set_symmetry(I64(nirrep), ptr(d))
    assert rc == 0


def desc(pops, iops, sym):
    d = ODesc()
    for k in range(4):
        for i in range(8):
            d.pop[k][i] = int(pops[k][i])
    d.iop[0], d.iop[1] = int(iops[0]), int(iops[1])
    d.sym = int(sym)
    return d


def desc_len(d):
    lib().o_desc_len.restype = I64
    return int(lib().o_desc_len(ctypes.byref(d)))


def vv2v_dpd(v1, d1, t1, v2, d2, t2, v3, d3, t3, f1, f2):
    rc = lib().o_vv2v_dpd(ptr(v1), ctypes.byref(d1), t1.encode(), ptr(v2), ctypes.byref(d2), t2.encode(),
                          ptr(v3), ctypes.byref(d3), t3.encode(), ctypes.c_double(f1), ctypes.c_double(f2))
    return rc


def opt(pops, iops, sym, arr):
    o = OOpt()
    o.d = desc(pops, iops, sym)
    o.arr = arr.ctypes.data
    o.len = arr.size
    return o


def call_kernel(name, out, a, b, fact):
    """Call an oracle lib_cc kernel o_<name>(out, a, b, fact) on OOpt views."""
    fn = getattr(lib(), "o_" + name)
    fn.restype = ctypes.c_int
    return fn(ctypes.byref(out), ctypes.byref(a), ctypes.byref(b), ctypes.c_double(fact))


def call_wrapper(name, v1, v2, v3, fact, t1, t2, t3, anti=None):
    fn = getattr(lib(), "o_" + name)
    fn.restype = ctypes.c_int
    args = [ctypes.byref(v1), ctypes.byref(v2), ctypes.byref(v3), ctypes.c_double(fact),
            t1.encode(), t2.encode(), t3.encode()]
    if anti is not None:
        args.append(I64(anti))
    return fn(*args)


def make_system(s):
    """OSystem from a synth.System (installs the symmetry table)."""
    o = OSystem()
    o.nirrep = s.nirrep
    for i in range(64):
        o.dirprd[i] = int(s.dirprd[i])
    o.symry = s.symry
    for k in range(8):
        o.popa[k], o.popb[k], o.vrta[k], o.vrtb[k] = int(s.popa[k]), int(s.popb[k]), int(s.vrta[k]), int(s.vrtb[k])
    rc = lib().o_system_init(ctypes.byref(o))
    assert rc == 0
    assert list(o.popo) == [int(x) for x in s.popo] and list(o.popv) == [int(x) for x in s.popv]
    return o


def make_integrals(s):
    I = OIntegrals()
    for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd"):
        setattr(I, k, s.ints[k].ctypes.data if s.ints[k] is not None else None)
    I.eorb = s.eorb.ctypes.data
    return I


def make_params(s, nthreads=1, **kw):
    p = OParams()
    lib().o_params_default(ctypes.byref(p))
    for h in range(8):
        p.estate_sym[h] = int(s.estate_sym[h])
    p.spin_flip = s.spin_flip
    p.nthreads = nthreads
    for k, v in {**getattr(s, 'run_opts', {}), **kw}.items():
        setattr(p, k, v)
    return p


def set_threads(n):
    lib().o_set_threads(I64(n))


class Oracle:
    """Stage-by-stage oracle run on a synth.System."""

    def __init__(self, s, nthreads=1, **params):
        self.s = s
        set_threads(nthreads)
        self.osys = make_system(s)
        self.oint = make_integrals(s)
        self.par = make_params(s, nthreads=nthreads, **params)

    def cis(self):
        s = self.s
        nroot = s.nroots
        rlen = sum(int(s.estate_sym[h]) * s.r1_len(h + 1) for h in range(8))
        om = np.zeros(max(nroot, 1))
        R = np.zeros(max(rlen, 1))
        it = I64(0)
        rc = lib().o_cis_run(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                             ptr(om), ptr(R), ctypes.byref(it))
        assert rc == 0, rc
        return om[:nroot], R[:rlen], it.value

    def cisdoo(self):
        """CIS(D-infinity) roots: omega and per root (R1, R2) of its irrep"""
        s = self.s
        nroot = s.nroots
        rlen = sum(int(s.estate_sym[h]) * (s.r1_len(h + 1) + s.r2_len(h + 1)) for h in range(8))
        om = np.zeros(max(nroot, 1))
        R = np.zeros(max(rlen, 1))
        it = I64(0)
        rc = lib().o_cisdoo_run(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                ptr(om), ptr(R), ctypes.byref(it))
        assert rc == 0, rc
        return om[:nroot], R[:rlen], it.value

    def ground(self):
        s = self.s
        l1, l2 = s.r1_len(1), s.r2_len(1)
        T2_1, T1_2, T2_2 = np.zeros(l2), np.zeros(l1), np.zeros(l2)
        E2, E3, it = ctypes.c_double(), ctypes.c_double(), I64()
        rc = lib().o_cpsd_ground(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                 ptr(T2_1), ptr(T1_2), ptr(T2_2), ctypes.byref(E2), ctypes.byref(E3),
                                 ctypes.byref(it))
        assert rc == 0, rc
        return dict(T2_1=T2_1, T1_2=T1_2, T2_2=T2_2, E2=E2.value, E3=E3.value, iters=it.value)

    def grcpsd(self):
        """grCPS(D) ground state: per order (T1, T2), E^(2..4), DIIS iterations"""
        s = self.s
        l1, l2 = s.r1_len(1), s.r2_len(1)
        T = np.zeros(3 * (l1 + l2))
        E = np.zeros(3)
        it = (I64 * 3)()
        rc = lib().o_grcpsd_ground(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                   ptr(T), ptr(E), it)
        assert rc == 0, rc
        T = T.reshape(3, l1 + l2)
        return dict(T1=[T[k, :l1] for k in range(3)], T2=[T[k, l1:] for k in range(3)], E=E,
                    iters=list(it))

    def eegrcpsd(self, g, om, R0):
        """EE-grCPS(D) of every root from grcpsd() and cisdoo() results:
        w (nroot x 3), left vectors and R^(1), R^(2) (cisdoo's layout)"""
        s = self.s
        nroot = s.nroots
        rlen = sum(int(s.estate_sym[h]) * (s.r1_len(h + 1) + s.r2_len(h + 1)) for h in range(8))
        T = np.concatenate([np.concatenate([g["T1"][k], g["T2"][k]]) for k in range(3)])
        w = np.zeros(3 * max(nroot, 1))
        L = np.zeros(max(rlen, 1))
        R = np.zeros(2 * max(rlen, 1))
        it = I64()
        om = np.ascontiguousarray(om, dtype=np.float64)
        R0 = np.ascontiguousarray(R0, dtype=np.float64)
        rc = lib().o_eegrcpsd_roots(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                    ptr(T), ptr(om), ptr(R0), ptr(w), ptr(L), ptr(R), ctypes.byref(it))
        assert rc == 0, rc
        return dict(w=w[:3 * nroot].reshape(nroot, 3), L=L[:rlen], R1=R[:rlen], R2=R[rlen:2 * rlen],
                    iters=it.value)

    def ground3(self, g):
        """third order ground state (run3.f90) from the T of ground()"""
        s = self.s
        l1, l2 = s.r1_len(1), s.r2_len(1)
        T1_3, T2_3 = np.zeros(l1), np.zeros(l2)
        E4, it = ctypes.c_double(), I64()
        rc = lib().o_cpsd_ground3(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                  ptr(g["T2_1"]), ptr(g["T1_2"]), ptr(g["T2_2"]), ptr(T1_3), ptr(T2_3),
                                  ctypes.byref(E4), ctypes.byref(it))
        assert rc == 0, rc
        return dict(T1_3=T1_3, T2_3=T2_3, E4=E4.value, iters=it.value)

    def jints(self, g):
        s, sym = self.s, self.s.sym
        o, v = s.popo, s.popv
        J = {
            "J2_Foo": np.zeros(sym.irpdso(1, o, o, 1)), "J2_Fvv": np.zeros(sym.irpdso(1, v, v, 1)),
            "J2_Wovvo": np.zeros(sym.idsymsoc(1, v, o, 1, v, o, 1)),
            "J2_Wovoo": np.zeros(sym.idsymsoc(1, o, o, 0, o, v, 1)),
            "J3_Foo": np.zeros(sym.irpdso(1, o, o, 1)), "J3_Fvv": np.zeros(sym.irpdso(1, v, v, 1)),
            "J3_Wovvo": np.zeros(sym.idsymsoc(1, v, o, 1, v, o, 1)),
        }
        oj = OJints()
        for k, a in J.items():
            setattr(oj, k, a.ctypes.data)
        rc = lib().o_calJ(ctypes.byref(self.osys), ctypes.byref(self.oint), ptr(g["T2_1"]), ptr(g["T1_2"]),
                          ptr(g["T2_2"]), ctypes.byref(oj))
        assert rc == 0, rc
        self._oj = oj
        return J

    def root(self, g, J, symR, w0, L):
        s = self.s
        oj = OJints()
        for k, a in J.items():
            setattr(oj, k, a.ctypes.data)
        l1, l2 = s.r1_len(symR), s.r2_len(symR)
        w = np.zeros(3)
        R2_1, R1_2, R2_2 = np.zeros(l2), np.zeros(l1), np.zeros(l2)
        it = I64()
        L = np.ascontiguousarray(L)
        rc = lib().o_eecpsd_root(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                 ptr(g["T2_1"]), ctypes.byref(oj), I64(symR), ctypes.c_double(w0), ptr(L),
                                 ptr(w), ptr(R2_1), ptr(R1_2), ptr(R2_2), ctypes.byref(it))
        assert rc == 0, rc
        return dict(w=w, R2_1=R2_1, R1_2=R1_2, R2_2=R2_2, iters=it.value)

    def pipeline(self):
        s = self.s
        n = max(s.nroots, 1)
        om, w2, w3 = np.zeros(n), np.zeros(n), np.zeros(n)
        nr = I64()
        rc = lib().o_sfcpsd_pipeline(ctypes.byref(self.osys), ctypes.byref(self.oint), ctypes.byref(self.par),
                                     ptr(om), ptr(w2), ptr(w3), ctypes.byref(nr))
        assert rc == 0, rc
        return om[:nr.value], w2[:nr.value], w3[:nr.value]
