"""The readers and writers of the reference's input files (host only, no
GPU): DPD lists (clmoioso0.f:30-67, updmoiso.f:50-75, getlstso.f:50-125,
getallso_d.f:31-79) and the interface node file
(src/pyscf2cc/mod_interface.f90).  The bytes are checked against an
independent parse written from those sources here (gfortran layout with
8-byte integers: 4-byte record markers around every sequential record,
32768-byte direct-access records; stream interface file with a 16-byte
header and 36-byte nodes), and a synthetic molecule's whole input
(c2v_nmo48) round-trips through the files bit for bit."""
import struct

import numpy as np
import pytest

from cpsd_b200 import api, synth

REC = 32768


def seq_records(path):
    """the records of a sequential unformatted file (4-byte markers)"""
    data = open(path, "rb").read()
    out, p = [], 0
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        out.append(data[p + 4:p + 4 + n])
        (m,) = struct.unpack_from("<i", data, p + 4 + n)
        assert m == n
        p += 8 + n
    return out


def i64s(b):
    return np.frombuffer(b, dtype="<i8")


@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_dpd_list_bytes_and_round_trip(tmp_path, nirrep):
    s = synth.System(nmo=40, nocc_a=5, nocc_b=3, nirrep=nirrep, seed=nirrep, skip_abcd=True)
    api.init(s.nirrep, s.dirprd)
    o, v = s.popo, s.popv
    cases = [("abci_ns_", [v, v, v, o], (0, 1), 1), ("iabj_ns_", [v, o, v, o], (1, 1), 1),
             ("ttmp1___", [v, v, o, o], (0, 0), 2 if nirrep > 1 else 1)]
    for name, pops, iops, sym in cases:
        n = s.sym.idsymsoc(sym, pops[0], pops[1], iops[0], pops[2], pops[3], iops[1])
        x = np.random.default_rng(n).standard_normal(n)
        api.write_dpd_list(str(tmp_path), name, sym, pops, iops, x)
        fname = name
        recs = seq_records(str(tmp_path / (fname + ".c")))
        # clmoioso0.f:53-65: irrepx, popp..pops, ioppq, ioprs, irrepr, irrepi,
        # moionuml(10,20), moionumr(10,20), rectmp(10,20)
        assert [len(r) for r in recs] == [8] + [64] * 8 + [1600] * 3
        assert i64s(recs[0])[0] == sym
        for k in range(4):
            np.testing.assert_array_equal(i64s(recs[1 + k]), pops[k])
        assert i64s(recs[5])[0] == iops[0] and i64s(recs[6])[0] == iops[1] and i64s(recs[7])[0] == sym
        numl = i64s(recs[9]).reshape(20, 10)[0]
        numr = i64s(recs[10]).reshape(20, 10)[0]
        rect = i64s(recs[11]).reshape(20, 10)
        raw = open(str(tmp_path / fname), "rb").read()
        assert len(raw) % REC == 0
        got, recs_used = [], 0
        for R in range(1, s.nirrep + 1):
            L = s.sym.dp(R, sym)
            nl = s.sym.irpdso(L, pops[0], pops[1], iops[0])
            nr = s.sym.irpdso(R, pops[2], pops[3], iops[1])
            assert numl[R - 1] == nl and numr[R - 1] == nr
            # updmoiso.f: each block starts on a record, after the previous one
            assert rect[0][R - 1] == recs_used
            got.append(np.frombuffer(raw, dtype="<f8", count=nl * nr, offset=REC * recs_used))
            recs_used += -(-(nl * nr) // (REC // 8))
        assert rect[1][0] == recs_used and len(raw) == REC * recs_used
        np.testing.assert_array_equal(np.concatenate(got), x)
        np.testing.assert_array_equal(api.read_dpd_list(str(tmp_path), name, n), x)
        with pytest.raises(api.CpsdError, match="elements"):
            api.read_dpd_list(str(tmp_path), name, n + 1)


def test_interface_node_file(tmp_path):
    path = str(tmp_path / "interface")
    a = np.arange(5, dtype=np.float64) * 0.5
    api.interface_write(path, "Orb_Energy", a)
    api.interface_write(path, "nirrep", np.array([4], dtype=np.int64))
    api.interface_write(path, "group_n", np.frombuffer(b"C2v", dtype=np.uint8))
    raw = open(path, "rb").read()
    meta, nnode = struct.unpack_from("<qq", raw, 0)
    # get_node: data from byte 17 on, each node at the old table position
    assert nnode == 3 and meta == 17 + 40 + 8 + 3
    nodes = []
    for i in range(nnode):
        rec = raw[meta - 1 + 36 * i: meta - 1 + 36 * (i + 1)]
        name = rec[:20].decode().rstrip(" ")
        pos, size = struct.unpack_from("<qq", rec, 20)
        nodes.append((name, pos, size))
    assert nodes == [("orb_energy", 17, 40), ("nirrep", 57, 8), ("group_n", 65, 3)]
    np.testing.assert_array_equal(np.frombuffer(raw, dtype="<f8", count=5, offset=16), a)
    np.testing.assert_array_equal(api.interface_read(path, "ORB_ENERGY"), a)
    # rewritten with the same size: in place; longer: behind the data
    api.interface_write(path, "nirrep", np.array([8], dtype=np.int64))
    assert api.interface_read(path, "nirrep", np.int64)[0] == 8
    assert struct.unpack_from("<qq", open(path, "rb").read(), 0) == (meta, 3)
    b = np.arange(7, dtype=np.float64)
    api.interface_write(path, "orb_energy", b)
    np.testing.assert_array_equal(api.interface_read(path, "orb_energy"), b)
    assert struct.unpack_from("<qq", open(path, "rb").read(), 0) == (meta + 56, 3)
    with pytest.raises(api.CpsdError, match="not found"):
        api.interface_read(path, "missing")


def test_synthetic_inputs_round_trip(tmp_path):
    """c2v_nmo48: the interface nodes and integral lists a run directory of
    the reference would hold, written and read back bit for bit"""
    s = synth.make("c2v_nmo48")
    ipath = str(tmp_path / "interface")
    api.write_inputs(str(tmp_path), ipath, s)
    sc = api.load_system(ipath)
    assert sc.nirrep == s.nirrep and sc.symry == s.symry
    assert list(sc.dirprd) == [int(x) for x in s.dirprd]
    for k in ("popa", "popb", "vrta", "vrtb"):
        assert list(getattr(sc, k)) == [int(x) for x in getattr(s, k)]
    got = api.load_inputs(str(tmp_path), ipath, sc, s.lengths(), len(s.eorb))
    for k in api.LIST_NAMES:
        np.testing.assert_array_equal(got[k], s.ints[k], err_msg=k)
    np.testing.assert_array_equal(got["eorb"], s.eorb)
    # the list directory from the interface's tmpdir node
    api.interface_write(ipath, "tmpdir", np.frombuffer(str(tmp_path).encode(), dtype=np.uint8))
    got2 = api.load_inputs(None, ipath, sc, s.lengths(), len(s.eorb))
    np.testing.assert_array_equal(got2["abcd"], s.ints["abcd"])
    # a list whose layout is not the programs' is refused
    api.write_dpd_list(str(tmp_path), "abij_ns_", 1, [s.popv, s.popv, s.popo, s.popo], (1, 1), np.zeros(
        s.sym.idsymsoc(1, s.popv, s.popv, 1, s.popo, s.popo, 1)))
    with pytest.raises(api.CpsdError, match="iops"):
        api.load_inputs(str(tmp_path), ipath, sc, s.lengths(), len(s.eorb))


def test_orbital_map_matches_spin_orbital_order():
    """api.orbital_map (the (mo, spin) map of cpsd_eri_lists /
    cpsd_eri_adjoint) lists the spin-free orbitals in the DPD lists' order,
    the order of the independent dense reference."""
    import dense
    from cpsd_b200 import api, synth
    for nirrep in (1, 2, 4, 8):
        s = synth.System(nmo=16 if nirrep < 8 else 24, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=1)
        mo, sp = api.orbital_map(s)
        occ, vir = dense.spin_orbitals(s)
        assert list(zip(mo.tolist(), sp.tolist())) == occ + vir
        assert len(mo) == int(sum(s.popo) + sum(s.popv))
