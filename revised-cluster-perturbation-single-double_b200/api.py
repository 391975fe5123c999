"""Python binding of libcpsd_b200 (the C-ABI in include/cpsd_b200.h).

Mirrors the reference's call surface for the SF-CIS / SF-CPS(D-3) path:
vv2v_dpd_444/424/442/422/222 (src/libsrint/vv2v_dpd_*.f90), the opt-level
contraction wrappers (src/lib_cc/mod_contract.f90), the spin-free lib_cc
kernels (src/lib_cc/<name>.f90) and the program drivers (EE-CIS.SF,
CPSd.SF, EE-CPSd.SF).  Device memory comes from torch CUDA tensors; torch is
plumbing only.  Every call raises CpsdError on a non-zero return code.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libcpsd_b200.so")
I64 = ctypes.c_int64
_lib = None


class CpsdError(RuntimeError):
    pass


def lib():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CpsdError(f"CUDA library missing: {LIB_PATH} (run __graft_entry__.build())")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.cpsd_last_error.restype = ctypes.c_char_p
        _lib.cpsd_launch_count.restype = I64
        _lib.cpsd_flop_count.restype = ctypes.c_double
        _lib.cpsd_workspace_high_water.restype = ctypes.c_size_t
        for f in ("cpsd_irpdso", "cpsd_idsymsoc", "cpsd_isymoffso"):
            getattr(_lib, f).restype = I64
    return _lib


def check(rc, what=""):
    if rc != 0:
        msg = lib().cpsd_last_error().decode(errors="replace")
        raise CpsdError(f"{what} failed with code {rc}: {msg}")
    return rc


class Opt(ctypes.Structure):
    """POD mirror of type(opt) (src/lib_cc/mod_operator.f90:8-25)."""
    _fields_ = [("popp", I64 * 8), ("popq", I64 * 8), ("popr", I64 * 8), ("pops", I64 * 8),
                ("ioppq", I64), ("ioprs", I64), ("sym", I64), ("len", I64), ("arr", ctypes.c_void_p)]


class System(ctypes.Structure):
    _fields_ = [("nirrep", I64), ("dirprd", I64 * 64), ("symry", I64),
                ("popa", I64 * 8), ("popb", I64 * 8), ("vrta", I64 * 8), ("vrtb", I64 * 8)]


class Integrals(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb")]


class Params(ctypes.Structure):
    _fields_ = [("davidson_dim", I64), ("davidson_cyc", I64), ("davidson_conv", I64), ("lowest", I64),
                ("diis_dim", I64), ("diis_cyc", I64), ("diis_max_err", ctypes.c_double),
                ("spin_flip", I64), ("open_shell", I64), ("ex_mult", I64), ("estate_sym", I64 * 8),
                ("batch_roots", I64)]


class Jints(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("J2_Foo", "J2_Fvv", "J2_Wovvo", "J2_Wovoo",
                                               "J3_Foo", "J3_Fvv", "J3_Wovvo")]


def arr8(v):
    return (I64 * 8)(*[int(x) for x in v])


def dptr(t):
    """device pointer of a torch CUDA tensor (or None)"""
    if t is None:
        return None
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise CpsdError("expected a contiguous float64 CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


def init(nirrep, dirprd):
    d = np.ascontiguousarray(dirprd, dtype=np.int64)
    check(lib().cpsd_init(I64(nirrep), d.ctypes.data_as(ctypes.c_void_p)), "cpsd_init")


def use_torch_stream():
    import torch
    check(lib().cpsd_set_stream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "cpsd_set_stream")


def launch_count(reset=False):
    return int(lib().cpsd_launch_count(1 if reset else 0))


def flop_count(reset=False):
    """useful contraction flops issued since the last reset"""
    return float(lib().cpsd_flop_count(1 if reset else 0))


def set_mixed(digits, min_gflop=1.0):
    """int8-digit tensor-core contractions with `digits` 7-bit digits per
    FP64 value for contractions of at least min_gflop GFLOP (0 = off)"""
    check(lib().cpsd_set_mixed(ctypes.c_int(digits), ctypes.c_double(min_gflop)), "cpsd_set_mixed")


def mixed_error(reset=True):
    """1 if a bounded wait of the digit path timed out since the last reset"""
    rc = lib().cpsd_mixed_error(ctypes.c_int(1 if reset else 0))
    if rc < 0:
        check(rc, "cpsd_mixed_error")
    return rc


def contract_records(maxrec=16384):
    """Per-launch records of the contraction timing buffer (timing must
    have been on, see contract_timing): milliseconds, useful flops, kind
    (0-3 FP64 tile shapes, 10/11 digit slicing, 12 digit GEMM, 20/21 narrow,
    30/31 Davidson, 32 solver, 40 pair transform) and size triple."""
    ms, fl = np.zeros(maxrec), np.zeros(maxrec)
    sh = np.zeros(4 * maxrec, np.int64)
    nr = I64()
    check(lib().cpsd_contract_records(ms.ctypes.data_as(ctypes.c_void_p), fl.ctypes.data_as(ctypes.c_void_p),
                                      sh.ctypes.data_as(ctypes.c_void_p), I64(maxrec), ctypes.byref(nr)),
          "cpsd_contract_records")
    k = nr.value
    shape = sh[:4 * k].reshape(k, 4)
    return ms[:k], fl[:k], shape[:, 3], shape[:, :3]


def contract_timing(on=True, reset=True):
    """per-launch CUDA-event timing of the library's kernels on/off"""
    check(lib().cpsd_contract_timing(ctypes.c_int(1 if on else 0)), "cpsd_contract_timing")
    if reset:
        check(lib().cpsd_contract_time(None, None, None, ctypes.c_int(1)), "cpsd_contract_time")


def set_tile_autotune(on=True):
    """empirical tile-shape choice of the FP64 tile kernel on / off"""
    check(lib().cpsd_set_tile_autotune(ctypes.c_int(1 if on else 0)), "cpsd_set_tile_autotune")


def tile_autotune_stats():
    """(plans tuned, plans whose tile shape the tuning changed)"""
    a, b = I64(), I64()
    check(lib().cpsd_tile_autotune_stats(ctypes.byref(a), ctypes.byref(b)), "cpsd_tile_autotune_stats")
    return a.value, b.value


def davidson_stats(reset=True):
    """(steps that solved the general non-symmetric Ritz problem, complex Ritz
    values met) on this thread since the last reset"""
    a, b = I64(), I64()
    check(lib().cpsd_davidson_stats(ctypes.byref(a), ctypes.byref(b), 1 if reset else 0), "cpsd_davidson_stats")
    return a.value, b.value


def geev(A):
    """The Davidson step's general eigen-solve on a host matrix (n <= 32):
    (wr, wi, V, sweeps) with dgeev's eigenvector columns in V."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    wr, wi, V = np.zeros(n), np.zeros(n), np.zeros((n, n))
    sw = I64()
    check(lib().cpsd_debug_geev(A.ctypes.data_as(ctypes.c_void_p), I64(n), wr.ctypes.data_as(ctypes.c_void_p),
                                wi.ctypes.data_as(ctypes.c_void_p), V.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(sw)), "cpsd_debug_geev")
    return wr, wi, V, sw.value


def opt(pops, iops, sym, t):
    o = Opt()
    check(lib().cpsd_opt_init(ctypes.byref(o), arr8(pops[0]), arr8(pops[1]), arr8(pops[2]), arr8(pops[3]),
                              I64(iops[0]), I64(iops[1]), I64(sym), dptr(t)), "cpsd_opt_init")
    return o


def kernel(name, out, a, b, fact=1.0):
    """cpsd_<name>(out, a, b, fact): one of the lib_cc kernels on Opt views."""
    fn = getattr(lib(), "cpsd_" + name)
    check(fn(ctypes.byref(out), ctypes.byref(a), ctypes.byref(b), ctypes.c_double(fact)), name)


def vv2v_dpd_444(v1, d1, t1, v2, d2, t2, v3, d3, t3, f1, f2):
    """vv2v_dpd_444 on device tensors; dK = (pops[4], iops[2], sym)."""
    (p1, i1, s1), (p2, i2, s2), (p3, i3, s3) = d1, d2, d3
    check(lib().cpsd_vv2v_dpd_444(
        dptr(v1), arr8(p1[0]), arr8(p1[1]), I64(i1[0]), arr8(p1[2]), arr8(p1[3]), I64(i1[1]), I64(s1), t1.encode(),
        dptr(v2), arr8(p2[0]), arr8(p2[1]), I64(i2[0]), arr8(p2[2]), arr8(p2[3]), I64(i2[1]), I64(s2), t2.encode(),
        dptr(v3), arr8(p3[0]), arr8(p3[1]), I64(i3[0]), arr8(p3[2]), arr8(p3[3]), I64(i3[1]), I64(s3), t3.encode(),
        ctypes.c_double(f1), ctypes.c_double(f2)), "vv2v_dpd_444")


def vv2v_dpd_444_noalloc(v1, d1, t1, v2, d2, t2, v3, d3, t3, f1, f2):
    """vv2v_dpd_444 through the entry point that allocates no device memory
    (tables and split-K partials in the library's fixed 32 MiB region)."""
    (p1, i1, s1), (p2, i2, s2), (p3, i3, s3) = d1, d2, d3
    check(lib().cpsd_vv2v_dpd_444_noalloc(
        dptr(v1), arr8(p1[0]), arr8(p1[1]), I64(i1[0]), arr8(p1[2]), arr8(p1[3]), I64(i1[1]), I64(s1), t1.encode(),
        dptr(v2), arr8(p2[0]), arr8(p2[1]), I64(i2[0]), arr8(p2[2]), arr8(p2[3]), I64(i2[1]), I64(s2), t2.encode(),
        dptr(v3), arr8(p3[0]), arr8(p3[1]), I64(i3[0]), arr8(p3[2]), arr8(p3[3]), I64(i3[1]), I64(s3), t3.encode(),
        ctypes.c_double(f1), ctypes.c_double(f2)), "vv2v_dpd_444_noalloc")


def make_system(s):
    """System struct from a synth.System (or any object with the same fields)."""
    o = System()
    o.nirrep = s.nirrep
    for i in range(64):
        o.dirprd[i] = int(s.dirprd[i])
    o.symry = s.symry
    for k in range(8):
        o.popa[k], o.popb[k], o.vrta[k], o.vrtb[k] = int(s.popa[k]), int(s.popb[k]), int(s.vrta[k]), int(s.vrtb[k])
    return o


def make_params(s, batch_roots=1, **kw):
    p = Params()
    lib().cpsd_params_default(ctypes.byref(p))
    for h in range(8):
        p.estate_sym[h] = int(s.estate_sym[h])
    p.spin_flip = s.spin_flip
    p.batch_roots = batch_roots
    for k, v in {**getattr(s, 'run_opts', {}), **kw}.items():
        setattr(p, k, v)
    return p


class DeviceIntegrals:
    """The six spin-free integral tensors and Eorb resident in HBM."""

    KEYS = ("ijkl", "ijka", "abij", "iabj", "abci", "abcd")

    def __init__(self, s, device="cuda"):
        import torch
        self.t = {}
        for k in self.KEYS:
            a = s.ints[k]
            self.t[k] = torch.from_numpy(a).to(device) if a is not None else None
        self.t["eorb"] = torch.from_numpy(s.eorb).to(device)
        self.struct = Integrals()
        for k, v in self.t.items():
            setattr(self.struct, k, v.data_ptr() if v is not None else None)

    @classmethod
    def from_tensors(cls, t):
        """wrap a dict of device tensors (ijkl ... abcd, eorb; missing: NULL)"""
        self = cls.__new__(cls)
        self.t = {k: t.get(k) for k in cls.KEYS}
        self.t["eorb"] = t["eorb"]
        self.struct = Integrals()
        for k, v in self.t.items():
            setattr(self.struct, k, v.data_ptr() if v is not None else None)
        return self

    @property
    def nbytes(self):
        return sum(v.numel() * 8 for v in self.t.values() if v is not None)


def cis_run(s, sysc, ints, par):
    import torch
    n = s.nroots
    rlen = sum(int(s.estate_sym[h]) * s.r1_len(h + 1) for h in range(8))
    om = np.zeros(max(n, 1))
    R = torch.zeros(max(rlen, 1), dtype=torch.float64, device="cuda")
    it = I64()
    check(lib().cpsd_cis_run(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par),
                             om.ctypes.data_as(ctypes.c_void_p), dptr(R), ctypes.byref(it)), "cpsd_cis_run")
    return om[:n], R[:rlen], it.value


def cisdoo_run(s, sysc, ints, par):
    """CIS(D-infinity): omega and per root (R1, R2) of its irrep (device)"""
    import torch
    n = s.nroots
    rlen = sum(int(s.estate_sym[h]) * (s.r1_len(h + 1) + s.r2_len(h + 1)) for h in range(8))
    om = np.zeros(max(n, 1))
    R = torch.zeros(max(rlen, 1), dtype=torch.float64, device="cuda")
    it = I64()
    check(lib().cpsd_cisdoo_run(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par),
                                om.ctypes.data_as(ctypes.c_void_p), dptr(R), ctypes.byref(it)), "cpsd_cisdoo_run")
    return om[:n], R[:rlen], it.value


def ground(s, sysc, ints, par):
    import torch
    l1, l2 = s.r1_len(1), s.r2_len(1)
    T2_1 = torch.zeros(l2, dtype=torch.float64, device="cuda")
    T1_2 = torch.zeros(l1, dtype=torch.float64, device="cuda")
    T2_2 = torch.zeros(l2, dtype=torch.float64, device="cuda")
    E2, E3, it = ctypes.c_double(), ctypes.c_double(), I64()
    check(lib().cpsd_ground(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par), dptr(T2_1),
                            dptr(T1_2), dptr(T2_2), ctypes.byref(E2), ctypes.byref(E3), ctypes.byref(it)),
          "cpsd_ground")
    return dict(T2_1=T2_1, T1_2=T1_2, T2_2=T2_2, E2=E2.value, E3=E3.value, iters=it.value)


def grcpsd_ground(s, sysc, ints, par):
    """grCPS(D) ground state: per order (T1, T2) on the device, E^(2..4), DIIS iterations"""
    import torch
    l1, l2 = s.r1_len(1), s.r2_len(1)
    T = torch.zeros(3 * (l1 + l2), dtype=torch.float64, device="cuda")
    E = np.zeros(3)
    it = (I64 * 3)()
    check(lib().cpsd_grcpsd_ground(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par), dptr(T),
                                   E.ctypes.data_as(ctypes.c_void_p), it), "cpsd_grcpsd_ground")
    T = T.view(3, l1 + l2)
    return dict(T1=[T[k, :l1] for k in range(3)], T2=[T[k, l1:] for k in range(3)], E=E, iters=list(it))


def eegrcpsd_roots(s, sysc, ints, par, g, om, R0):
    """EE-grCPS(D) of every root from grcpsd_ground() and cisdoo_run()
    results: w (nroot x 3), left vectors, R^(1), R^(2) (device), iterations"""
    import torch
    n = s.nroots
    rlen = sum(int(s.estate_sym[h]) * (s.r1_len(h + 1) + s.r2_len(h + 1)) for h in range(8))
    T = torch.cat([torch.cat([g["T1"][k], g["T2"][k]]) for k in range(3)]).contiguous()
    w = np.zeros(3 * max(n, 1))
    L = torch.zeros(max(rlen, 1), dtype=torch.float64, device="cuda")
    R = torch.zeros(2 * max(rlen, 1), dtype=torch.float64, device="cuda")
    it = I64()
    om = np.ascontiguousarray(om, dtype=np.float64)
    check(lib().cpsd_eegrcpsd_roots(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par), dptr(T),
                                    om.ctypes.data_as(ctypes.c_void_p), dptr(R0), w.ctypes.data_as(ctypes.c_void_p),
                                    dptr(L), dptr(R), ctypes.byref(it)), "cpsd_eegrcpsd_roots")
    return dict(w=w[:3 * n].reshape(n, 3), L=L[:rlen], R1=R[:rlen], R2=R[rlen:2 * rlen], iters=it.value)


def ground3(s, sysc, ints, par, g):
    """third-order ground state (run3.f90) from ground()'s T: T1^(3),
    T2^(3) (device) and E^(4)"""
    import torch
    l1, l2 = s.r1_len(1), s.r2_len(1)
    T1_3 = torch.zeros(l1, dtype=torch.float64, device="cuda")
    T2_3 = torch.zeros(l2, dtype=torch.float64, device="cuda")
    E4, it = ctypes.c_double(), I64()
    check(lib().cpsd_ground3(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par), dptr(g["T2_1"]),
                             dptr(g["T1_2"]), dptr(g["T2_2"]), dptr(T1_3), dptr(T2_3), ctypes.byref(E4),
                             ctypes.byref(it)), "cpsd_ground3")
    return dict(T1_3=T1_3, T2_3=T2_3, E4=E4.value, iters=it.value)


def calJ(s, sysc, ints, g):
    import torch
    sym, o, v = s.sym, s.popo, s.popv
    sizes = {"J2_Foo": sym.irpdso(1, o, o, 1), "J2_Fvv": sym.irpdso(1, v, v, 1),
             "J2_Wovvo": sym.idsymsoc(1, v, o, 1, v, o, 1), "J2_Wovoo": sym.idsymsoc(1, o, o, 0, o, v, 1),
             "J3_Foo": sym.irpdso(1, o, o, 1), "J3_Fvv": sym.irpdso(1, v, v, 1),
             "J3_Wovvo": sym.idsymsoc(1, v, o, 1, v, o, 1)}
    J = {k: torch.zeros(n, dtype=torch.float64, device="cuda") for k, n in sizes.items()}
    js = Jints()
    for k, t in J.items():
        setattr(js, k, t.data_ptr())
    check(lib().cpsd_calJ(ctypes.byref(sysc), ctypes.byref(ints.struct), dptr(g["T2_1"]), dptr(g["T1_2"]),
                          dptr(g["T2_2"]), ctypes.byref(js)), "cpsd_calJ")
    return J, js


def eecpsd_roots(s, sysc, ints, par, g, js, symR, w0, L, want_vectors=False):
    import torch
    nroot = len(w0)
    l1, l2 = s.r1_len(symR), s.r2_len(symR)
    w = np.zeros(3 * nroot)
    w0a = np.ascontiguousarray(w0, dtype=np.float64)
    outs = {}
    if want_vectors:
        outs = {"R2_1": torch.zeros(nroot * l2, dtype=torch.float64, device="cuda"),
                "R1_2": torch.zeros(nroot * l1, dtype=torch.float64, device="cuda"),
                "R2_2": torch.zeros(nroot * l2, dtype=torch.float64, device="cuda")}
    it = I64()
    check(lib().cpsd_eecpsd_roots(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par),
                                  dptr(g["T2_1"]), ctypes.byref(js), I64(symR), I64(nroot),
                                  w0a.ctypes.data_as(ctypes.c_void_p), dptr(L), w.ctypes.data_as(ctypes.c_void_p),
                                  dptr(outs.get("R2_1")), dptr(outs.get("R1_2")), dptr(outs.get("R2_2")),
                                  ctypes.byref(it)), "cpsd_eecpsd_roots")
    return w.reshape(nroot, 3), outs, it.value


def pipeline(s, sysc, ints, par):
    n = max(s.nroots, 1)
    om, w2, w3 = np.zeros(n), np.zeros(n), np.zeros(n)
    nr = I64()
    check(lib().cpsd_pipeline(ctypes.byref(sysc), ctypes.byref(ints.struct), ctypes.byref(par),
                              om.ctypes.data_as(ctypes.c_void_p), w2.ctypes.data_as(ctypes.c_void_p),
                              w3.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nr)), "cpsd_pipeline")
    return om[:nr.value], w2[:nr.value], w3[:nr.value]


class IntegralGrads(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb")]


def integrals_struct(t):
    """Integrals struct from a dict of float64 CUDA tensors (missing keys: NULL)."""
    st = Integrals()
    for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb"):
        v = t.get(k)
        p = dptr(v)
        setattr(st, k, p.value if p is not None else None)
    return st


def orbital_map(s):
    """(mo, spin) of every spin-free orbital of a synth.System in the DPD
    lists' order: per irrep the alpha then the beta occupied orbitals, then
    the virtual ones likewise"""
    occ, vir = [], []
    for h in range(1, s.nirrep + 1):
        for spin, nocc in ((0, s.nocc_a), (1, s.nocc_b)):
            occ += [(m, spin) for m in range(s.nmo) if s.mo_irrep[m] == h and m < nocc]
        for spin, nocc in ((0, s.nocc_a), (1, s.nocc_b)):
            vir += [(m, spin) for m in range(s.nmo) if s.mo_irrep[m] == h and m >= nocc]
    mo = np.array([m for m, _ in occ + vir], np.int64)
    sp = np.array([x for _, x in occ + vir], np.int64)
    return mo, sp


def eri_lists(sysc, orb_mo, orb_spin, nmo, eri, lists):
    """cpsd_eri_lists: fill the device lists (dict name -> tensor) from the
    dense (pq|rs) tensor eri (nmo^4, device)"""
    orb_mo = np.ascontiguousarray(orb_mo, np.int64)
    orb_spin = np.ascontiguousarray(orb_spin, np.int64)
    check(lib().cpsd_eri_lists(ctypes.byref(sysc), orb_mo.ctypes.data_as(ctypes.c_void_p),
                               orb_spin.ctypes.data_as(ctypes.c_void_p), I64(nmo), dptr(eri),
                               ctypes.byref(integrals_struct(lists))), "cpsd_eri_lists")


def eri_adjoint(sysc, orb_mo, orb_spin, nmo, grads, geri):
    """cpsd_eri_adjoint: geri (nmo^4, device) += d/d(pq|rs) of sum g.list"""
    orb_mo = np.ascontiguousarray(orb_mo, np.int64)
    orb_spin = np.ascontiguousarray(orb_spin, np.int64)
    check(lib().cpsd_eri_adjoint(ctypes.byref(sysc), orb_mo.ctypes.data_as(ctypes.c_void_p),
                                 orb_spin.ctypes.data_as(ctypes.c_void_p), I64(nmo),
                                 ctypes.byref(integrals_struct(grads)), dptr(geri)), "cpsd_eri_adjoint")


def cisd_energies(s, sysc, ints_struct, par, symR, nroot):
    """SF-CIS roots of irrep symR and their w^(2): (w0, w2, L) with L the
    unit CIS vectors (nroot x lenR1, CUDA)."""
    import torch
    l1 = s.r1_len(symR)
    L = torch.zeros(nroot * l1, dtype=torch.float64, device="cuda")
    w0, w2 = np.zeros(nroot), np.zeros(nroot)
    check(lib().cpsd_cisd_energies(ctypes.byref(sysc), ctypes.byref(ints_struct), ctypes.byref(par), I64(symR),
                                   I64(nroot), w0.ctypes.data_as(ctypes.c_void_p),
                                   w2.ctypes.data_as(ctypes.c_void_p), dptr(L)), "cpsd_cisd_energies")
    return w0, w2, L


def cisd_gradient(sysc, ints_struct, par, symR, w0, L, g0, g2, grads):
    """Adds d(sum g0 w0 + g2 w2) to grads (dict of CUDA tensors: ijka, abij,
    iabj, abci, eorb)."""
    w0 = np.ascontiguousarray(w0, dtype=np.float64)
    g0 = np.ascontiguousarray(g0, dtype=np.float64)
    g2 = np.ascontiguousarray(g2, dtype=np.float64)
    G = IntegralGrads()
    for k in ("ijka", "abij", "iabj", "abci", "eorb"):
        setattr(G, k, dptr(grads[k]).value)
    check(lib().cpsd_cisd_gradient(ctypes.byref(sysc), ctypes.byref(ints_struct), ctypes.byref(par), I64(symR),
                                   I64(len(w0)), w0.ctypes.data_as(ctypes.c_void_p), dptr(L),
                                   g0.ctypes.data_as(ctypes.c_void_p), g2.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.byref(G)), "cpsd_cisd_gradient")


def cpsd3_energies(s, sysc, ints_struct, par, symR, nroot):
    """SF-CIS roots of irrep symR with their w^(2) and w^(3): (w0, w2, w3, L),
    L the unit CIS vectors (nroot x lenR1, CUDA)."""
    import torch
    l1 = s.r1_len(symR)
    L = torch.zeros(nroot * l1, dtype=torch.float64, device="cuda")
    w0, w2, w3 = np.zeros(nroot), np.zeros(nroot), np.zeros(nroot)
    check(lib().cpsd_cpsd3_energies(ctypes.byref(sysc), ctypes.byref(ints_struct), ctypes.byref(par), I64(symR),
                                    I64(nroot), w0.ctypes.data_as(ctypes.c_void_p),
                                    w2.ctypes.data_as(ctypes.c_void_p), w3.ctypes.data_as(ctypes.c_void_p),
                                    dptr(L)), "cpsd_cpsd3_energies")
    return w0, w2, w3, L


def cpsd3_gradient(sysc, ints_struct, par, symR, w0, L, g0, g2, g3, grads):
    """Adds d(sum g0 w0 + g2 w2 + g3 w3) to grads (dict of CUDA tensors: all
    six lists and eorb)."""
    w0, g0, g2, g3 = (np.ascontiguousarray(x, dtype=np.float64) for x in (w0, g0, g2, g3))
    G = IntegralGrads()
    for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb"):
        setattr(G, k, dptr(grads[k]).value)
    check(lib().cpsd_cpsd3_gradient(ctypes.byref(sysc), ctypes.byref(ints_struct), ctypes.byref(par), I64(symR),
                                    I64(len(w0)), w0.ctypes.data_as(ctypes.c_void_p), dptr(L),
                                    g0.ctypes.data_as(ctypes.c_void_p), g2.ctypes.data_as(ctypes.c_void_p),
                                    g3.ctypes.data_as(ctypes.c_void_p), ctypes.byref(G)), "cpsd_cpsd3_gradient")


def set_phase_overlap(on=True):
    """SF-CIS beside the ground state on two library worker streams (True,
    the default) or all phases in order on the caller's stream"""
    check(lib().cpsd_set_phase_overlap(1 if on else 0), "cpsd_set_phase_overlap")


def pipeline_batch(systems, ints_list, params, nworkers=4):
    """cpsd_pipeline_batch over independent molecules: systems (synth.System
    or compatible), their DeviceIntegrals and Params; returns per-molecule
    (omega_cis, w2, w3) lists."""
    n = len(systems)
    S = (System * n)(*[make_system(s) for s in systems])
    I = (Integrals * n)(*[d.struct for d in ints_list])
    P = (Params * n)(*params)
    counts = [int(sum(p.estate_sym[h] for h in range(8))) for p in params]
    tot = max(sum(counts), 1)
    om, w2, w3 = np.zeros(tot), np.zeros(tot), np.zeros(tot)
    nr = I64()
    check(lib().cpsd_pipeline_batch(I64(n), S, I, P, I64(nworkers), om.ctypes.data_as(ctypes.c_void_p),
                                    w2.ctypes.data_as(ctypes.c_void_p), w3.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(nr)), "cpsd_pipeline_batch")
    out, k = [], 0
    for c in counts:
        out.append((om[k:k + c], w2[k:k + c], w3[k:k + c]))
        k += c
    return out


def release_device_cache():
    """cpsd_release_device_cache: free the library's idle device buffers."""
    check(lib().cpsd_release_device_cache(), "cpsd_release_device_cache")


# ------------------------------------------------ the reference's input files
# DPD lists (getallso / clmoioso0 + putlstso) and the "interface" node file
# (src/pyscf2cc/mod_interface.f90), read and written on the host.
LIST_NAMES = {"ijkl": "ijkl_ns_", "ijka": "ijka_ns_", "abij": "abij_ns_", "iabj": "iabj_ns_",
              "abci": "abci_ns_", "abcd": "abcd_ns_"}


class DpdListMeta(ctypes.Structure):
    _fields_ = [("irrepx", I64), ("popp", I64 * 8), ("popq", I64 * 8), ("popr", I64 * 8), ("pops", I64 * 8),
                ("ioppq", I64 * 8), ("ioprs", I64 * 8), ("irrepr", I64 * 8), ("irrepi", I64 * 8),
                ("moionuml", (I64 * 10) * 20), ("moionumr", (I64 * 10) * 20), ("rectmp", (I64 * 10) * 20)]


def _b(x):
    return None if x is None else str(x).encode()


def write_dpd_list(dirname, name, irrepx, pops, iops, arr):
    a = np.ascontiguousarray(arr, dtype=np.float64)
    check(lib().cpsd_dpd_list_write(_b(dirname), _b(name), I64(irrepx), arr8(pops[0]), arr8(pops[1]), I64(iops[0]),
                                    arr8(pops[2]), arr8(pops[3]), I64(iops[1]), a.ctypes.data_as(ctypes.c_void_p)),
          "cpsd_dpd_list_write")


def read_dpd_list(dirname, name, n):
    out = np.zeros(n)
    check(lib().cpsd_dpd_list_read(_b(dirname), _b(name), out.ctypes.data_as(ctypes.c_void_p), I64(n)),
          "cpsd_dpd_list_read")
    return out


def read_dpd_list_meta(dirname, name):
    m = DpdListMeta()
    check(lib().cpsd_dpd_list_meta_read(_b(dirname), _b(name), ctypes.byref(m)), "cpsd_dpd_list_meta_read")
    return m


def interface_write(path, node, data):
    a = np.ascontiguousarray(data)
    check(lib().cpsd_interface_write(_b(path), _b(node), a.ctypes.data_as(ctypes.c_void_p), I64(a.nbytes)),
          "cpsd_interface_write")


def interface_read(path, node, dtype=np.float64):
    n = I64()
    check(lib().cpsd_interface_size(_b(path), _b(node), ctypes.byref(n)), "cpsd_interface_size")
    out = np.zeros(n.value // np.dtype(dtype).itemsize, dtype=dtype)
    check(lib().cpsd_interface_read(_b(path), _b(node), out.ctypes.data_as(ctypes.c_void_p), n), "cpsd_interface_read")
    return out


def load_system(interface_path):
    """cpsd_system from the interface file (readmodule)"""
    sc = System()
    check(lib().cpsd_load_system(_b(interface_path), ctypes.byref(sc)), "cpsd_load_system")
    return sc


def load_inputs(dirname, interface_path, sysc, lengths, neorb, keys=tuple(LIST_NAMES)):
    """the six integral lists and the spin-free orbital energies (loadSCF)
    into host arrays; lengths: DPD length per tensor name"""
    out = {k: np.zeros(lengths[k]) for k in keys}
    out["eorb"] = np.zeros(neorb)
    p = [out[k].ctypes.data_as(ctypes.c_void_p) if k in out else None for k in LIST_NAMES]
    check(lib().cpsd_load_inputs(_b(dirname), _b(interface_path), ctypes.byref(sysc), *p,
                                 out["eorb"].ctypes.data_as(ctypes.c_void_p)), "cpsd_load_inputs")
    return out


def write_inputs(dirname, interface_path, s, eps_alpha=None, eps_beta=None):
    """The files a synth.System's integrals would have in the reference's
    run directory: the interface nodes readmodule / loadSCF read (the keys
    py2cc.write_interface writes plus 'orb_energy_no_spin') and the six
    spin-free integral lists."""
    init(s.nirrep, s.dirprd)
    dirprd = np.ascontiguousarray(np.asarray(s.dirprd, dtype=np.int64).reshape(64))
    interface_write(interface_path, "dirprd", dirprd)
    interface_write(interface_path, "vrt", np.concatenate([s.vrta, s.vrtb]).astype(np.int64))
    interface_write(interface_path, "pop", np.concatenate([s.popa, s.popb]).astype(np.int64))
    for k, v in (("symrx", 1), ("symry", s.symry), ("symrz", 1), ("nirrep", s.nirrep),
                 ("iprcln", 32768), ("iprcwd", 4096), ("ichcsz", 4096)):
        interface_write(interface_path, k, np.array([v], dtype=np.int64))
    interface_write(interface_path, "orb_energy_no_spin", np.asarray(s.eorb, dtype=np.float64))
    o, v = s.popo, s.popv
    layout = {"ijkl": ([o, o, o, o], (0, 0)), "ijka": ([o, o, o, v], (0, 1)), "abij": ([v, v, o, o], (0, 0)),
              "iabj": ([v, o, v, o], (1, 1)), "abci": ([v, v, v, o], (0, 1)), "abcd": ([v, v, v, v], (0, 0))}
    for k, (pops, iops) in layout.items():
        if s.ints.get(k) is not None:
            write_dpd_list(dirname, LIST_NAMES[k], 1, pops, iops, s.ints[k])
