"""Particle restart and snapshot files, and the param.in importer (no GPU).

The record layout is pinned against bytes assembled here with ``struct`` from the
gfortran rules (4-byte markers; subrecords whose head marker is negated when more
follow and whose tail marker is negated when others precede), and the two particle
layouts against the WRITE statements of save_particle.f90:163-180 and
print_particle.f90:151-164 written out the same way.  The reference's Fortran cannot be
compiled here, so these byte layouts stand in for files it wrote."""
from __future__ import annotations

import os
import struct

import numpy as np
import pytest

from gazpart_b200 import _lib, params, restart
from gazpart_b200._lib import GPError


def rec(payload: bytes) -> bytes:
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def f64(*v) -> bytes:
    return struct.pack(f"<{len(v)}d", *v)


def i32(*v) -> bytes:
    return struct.pack(f"<{len(v)}i", *v)


def test_records_have_gfortran_markers(tmp_path):
    p = str(tmp_path / "a.bin")
    with restart.FortranFile(p, "w") as f:
        f.write(np.array([7], np.int32))
        f.write(np.array([1.5, -2.0, 3.25]))
        f.write(np.array([], np.float64))
        f.write(np.array([1, 2], np.int32), np.array([0.5]))    # one record, two items
    want = rec(i32(7)) + rec(f64(1.5, -2.0, 3.25)) + rec(b"") + rec(i32(1, 2) + f64(0.5))
    assert open(p, "rb").read() == want
    with restart.FortranFile(p) as f:
        assert f.record_size() == 4
        assert f.read(np.int32, 1)[0] == 7
        assert f.read(np.float64, 2).tolist() == [1.5, -2.0]     # rest of the record is passed over
        f.skip()                                                 # the empty record
        assert f.read_record(np.int32).tolist() == [1, 2, 0, 1071644672]
        with pytest.raises(GPError) as e:
            f.read(np.int32, 1)
        assert e.value.code == _lib.GP_EEOF


def test_long_records_split_into_signed_subrecords(tmp_path):
    p = str(tmp_path / "b.bin")
    data = np.arange(5, dtype=np.float64)                 # 40 bytes
    with restart.FortranFile(p, "w", max_subrecord=16) as f:
        f.write(data)
        f.write(data[:2])                                 # exactly one full subrecord
    raw = data.tobytes()
    want = (i32(-16) + raw[:16] + i32(16) + i32(-16) + raw[16:32] + i32(-16) + i32(8) + raw[32:] + i32(-8)
            + rec(raw[:16]))
    assert open(p, "rb").read() == want
    with restart.FortranFile(p) as f:
        assert f.record_size() == 40
        assert np.array_equal(f.read(np.float64, 5), data)
        assert np.array_equal(f.read_record(np.float64), data[:2])


def test_reading_past_a_record_and_damaged_files(tmp_path):
    p = str(tmp_path / "c.bin")
    with restart.FortranFile(p, "w") as f:
        f.write(np.array([1.0, 2.0]))
        f.write(np.array([3.0]))
    with restart.FortranFile(p) as f:
        with pytest.raises(GPError) as e:
            f.read(np.float64, 3)                         # 'I/O past end of record'
        assert e.value.code == _lib.GP_ERECORD
        assert f.read(np.float64, 1)[0] == 3.0            # the short record was consumed
    raw = open(p, "rb").read()
    bad = str(tmp_path / "d.bin")
    open(bad, "wb").write(raw[:-6])                       # cut inside the second record
    with restart.FortranFile(bad) as f:
        f.skip()
        with pytest.raises(GPError) as e:
            f.skip()
        assert e.value.code == _lib.GP_EIO
    open(bad, "wb").write(raw[:20] + i32(99) + raw[24:])  # tail marker disagrees with the head
    with restart.FortranFile(bad) as f:
        with pytest.raises(GPError) as e:
            f.skip()
        assert e.value.code == _lib.GP_ERECORD
    with pytest.raises(GPError) as e:
        restart.FortranFile(str(tmp_path / "missing.bin"))
    assert e.value.code == _lib.GP_EIO


def _cols(n, seed):
    rng = np.random.default_rng(seed)
    c = {k: rng.normal(size=n) for k in restart.PART_COLUMNS if k != "idp"}
    c["idp"] = rng.integers(1, 3, size=n).astype(np.int32)
    return c


def test_class_restart_layout_and_round_trip(tmp_path):
    n = 5
    cols = _cols(n, 1)
    tables = restart.ClassTables(npclass=[3, 2], rhop=[1000.0, 2500.0], emaj=[0.01, 0.01], apr=2.5)
    p = str(tmp_path / restart.part_file_name(1, 120))
    restart.write_part_class(p, cols, tables)
    want = rec(i32(n)) + rec(i32(3, 2)) + rec(f64(1000.0, 2500.0)) + rec(f64(0.01, 0.01)) + rec(f64(2.5))
    for k in restart.PART_COLUMNS:
        want += rec(np.asarray(cols[k], np.float64).tobytes())
    assert open(p, "rb").read() == want
    back, t2 = restart.read_part_class(p)
    for k in restart.PART_COLUMNS:
        assert np.array_equal(back[k], cols[k]), k
    assert back["idp"].dtype == np.int32
    assert np.array_equal(t2.npclass, tables.npclass) and np.array_equal(t2.rhop, tables.rhop)
    assert np.array_equal(t2.emaj, tables.emaj) and t2.apr == tables.apr


def test_empty_class_and_snapshot(tmp_path):
    tables = restart.default_tables(0, 0.01, 2.0, 1000.0)
    p = str(tmp_path / "part_p01.end")
    restart.write_part_class(p, {k: np.empty(0) for k in restart.PART_COLUMNS}, tables)
    back, t2 = restart.read_part_class(p)
    assert all(back[k].size == 0 for k in restart.PART_COLUMNS) and t2.npclass.tolist() == [0]
    cols = _cols(7, 2)
    s = str(tmp_path / "snap.bin")
    restart.write_snapshot(s, cols)
    assert open(s, "rb").read() == b"".join(rec(np.asarray(cols[k], np.float64).tobytes())
                                            for k in restart.PART_COLUMNS)
    back = restart.read_snapshot(s)
    for k in restart.PART_COLUMNS:
        assert np.array_equal(back[k], cols[k]), k


def test_isavepart1_reader_cannot_read_its_writer(tmp_path):
    n = 4
    c = _cols(n, 3)
    c.update({k: np.full(n, 0.5) for k in ("ufap", "vfap", "wfap")})
    p = str(tmp_path / "PART.bin")
    restart.write_part_multi(p, [c])
    raw = open(p, "rb").read()
    want = rec(i32(n)) + rec(np.asarray(c["idp"], np.int32).tobytes())
    for k in ("x", "y", "z", "u", "v", "w", "ufap", "vfap", "wfap"):
        want += rec(np.asarray(c[k], np.float64).tobytes())
    assert raw == want
    with pytest.raises(GPError) as e:
        restart.read_part_multi(p, 1)
    assert e.value.code in (_lib.GP_ERECORD, _lib.GP_EEOF)
    # a file in the reader's own layout reads back
    q = str(tmp_path / "PART.ini")
    with restart.FortranFile(q, "w") as f:
        f.write(np.array([n], np.int32))
        f.write(np.asarray(c["idp"], np.int32))
        f.write(np.zeros(n))
        for k in ("x", "y", "z", "u", "v", "w", "ufap", "vfap", "wfap", "qa", "qb", "qc", "qd", "ox", "oy", "oz"):
            f.write(np.asarray(c[k], np.float64))
    got = restart.read_part_multi(q, 1)[0]
    for k in ("x", "qd", "oz", "ufap"):
        assert np.array_equal(got[k], c[k])
    assert np.array_equal(got["idp"], c["idp"])


def test_file_names_follow_the_fortran_formats():
    assert restart.part_file_name(1, 250) == "part_p01_t00000250.bin"
    assert restart.part_file_name(12, 0) == "part_p12_t00000000.bin"
    assert restart.part_file_name(3, kind="end") == "part_p03.end"
    assert restart.part_file_name(3, kind="ini") == "part_p03.ini"
    assert restart.part_file_name(100, 123456789) == "part_p**_t********.bin"    # I2.2 / I8.8 overflow
    assert restart.snapshot_file_name(2, 40) == "postprocessing/part_p02_t00000040.bin"


def test_tables_and_particle_constants():
    t = restart.default_tables(10, 0.002, 3.0, 1000.0, polydisp=2, nq_np=1.5, rhoq_rhop=4.0)
    idp = restart.initial_idp(10, 2, 1.5)
    assert idp.tolist() == [1] * 4 + [2] * 6           # int(10 / 2.5) = 4 of index 1
    assert t.npclass.tolist() == [4, 6] and t.rhop.tolist() == [1000.0, 250.0]
    assert t.emaj.tolist() == [0.002, 0.002]
    t1 = restart.default_tables(10, 0.002, 3.0, 1000.0, polydisp=1, polydispmax=2)
    assert t1.npclass.tolist() == [10, 10] and t1.rhop.tolist() == [1000.0, 1000.0]
    pr = restart.props_from_tables(idp, t)
    a, b = 0.002, 0.002 / 3.0
    assert pr["ipxx"][0] == (b * b + b * b) / 5.0 and pr["ipzz"][0] == (a * a + b * b) / 5.0
    assert pr["rhop"][9] == 250.0 and pr["apr"][0] == 3.0
    with pytest.raises(ValueError):
        restart.props_from_tables(np.array([3]), t)


# A param.in in READPARAM's order, written for these tests (values of a small run)
def _param_text(dry_channel: bool, nig: int = 1) -> str:
    lines = ["!"] * 7 + ["0", "!", "48", "40", "32", "!", "2.0E-4", "300",
                         "!", "2", "0", ".false.", "5.0E-2", "0.08", "2.0", "6.0",
                         "!", ".false.", "0", "!", ".true."]
    if dry_channel:
        lines.append(".false.     ! dry channel")
    lines += [f"{nig}   ! classes", "2000", ".false.", "3", "2", "2", "0"]
    lines += ["!"] * 3 + [".false.", ".true.", "-----!---", "1", "!", ".false.", ".false.", "!",
                          ".false.", ".false.", ".false.", ".false.", ".false."]
    lines += ["!"] * 3 + ["10", "500", "1", "0", "2", "0", "0", "28", "1.3"]
    lines += ["!"] * 3 + ["6.283185307179586", "6.283185307179586", "3.14159", "1.0e-2", "1.205"]
    lines += ["!"] * 3 + ["1.43E-3", "1005.0", "0.010E+0"]
    lines += ["!"] * 3
    for k in range(nig):
        lines += [f"2 {1 - k}", "0.003", "2.5", "1000.0D0", "1.0, 0.0", "0.0", "1005.0", f"{1 + k}",
                  "0.5 1.0 4.0", "! ---"]
    lines += ["1.0", "0.0", "0.0", "!", ".false. 128"]
    return "\n".join(lines) + "\n"


def test_param_reader_order_and_adjustments():
    p = params.parse_param(_param_text(False, nig=2))
    assert (p.nx, p.ny, p.nz) == (48, 40, 32) and p.dtime_user == 2.0e-4 and p.ncyclemax == 300
    assert p.frozen_flow == 2 and p.steady is False and p.solve_part is True
    assert p.nig == 2 and p.npart_full == 2000 and p.interp_scheme == 3
    assert p.lxmax == 6.283185307179586 and p.lzmax == 3.14159 and p.visc == 1.0e-2
    assert p.fout1 == 300                                  # FOUT1 capped at NCYCLEMAX
    c1, c2 = p.classes
    assert c1.rhop_user == 1000.0 and (c1.ecp, c1.mup) == (1.0, 0.0)
    assert (c1.nq_np, c1.dq_dp, c1.rhoq_rhop) == (0.0, 1.0, 1.0)    # POLYDISP = 1 resets them
    assert (c2.polydisp, c2.nq_np, c2.rhoq_rhop) == (2, 0.5, 4.0)
    assert p.solve_collision is True and p.periodicity is True and p.kcut == 128.0
    s = p.setup(1)
    assert (s.nx, s.lz, s.rhof, s.dtime) == (48, 3.14159, 1.205, 2.0e-4)
    t = p.tables(2)
    assert t.polydisp == 2 and t.rhop.tolist() == [1000.0, 250.0]
    assert t.npclass.tolist() == [int(2000 / 1.5), 2000 - int(2000 / 1.5)]
    # written back out in the reader's layout, it reads the same
    q = params.parse_param(params.format_param(p))
    assert q.values == p.values and q.classes == p.classes


def test_param_file_layout_mismatch():
    text = _param_text(True)
    with pytest.raises(params.ParamError) as e:
        params.parse_param(text)                           # the reader takes '.false.' as NIG
    assert e.value.line == 29 and "Bad integer" in str(e.value)
    p = params.parse_param(text, layout="file")
    assert p.dry_channel is False and p.nig == 1 and p.npart_full == 2000


def test_list_directed_details():
    r = params._ListReader("1 2\n3, , 5 / 9\n7*1.5\n2*\n.TRUE. FOO\n")
    assert r.read("iii") == [1, 2, 3]                      # continues on the next record
    assert r.read("rrr") == [1.5] * 3
    assert r.read("ii") == [None, None]                    # r* gives nulls
    assert r.read("ll")[0] is True
    with pytest.raises(params.ParamError):
        params._ListReader("1.0\n").read("i")
    assert params._ListReader("3, , 5 / 9\n").read("iiii") == [3, None, 5, None]
    assert params._ListReader("1.0D-3 2.5+2 .5\n").read("rrr") == [1.0e-3, 250.0, 0.5]


# The reference's own param.in (source/param.in of the reference tree), named by the
# environment; the test is skipped where the reference tree is not at hand.
SHIPPED = os.environ.get("GAZPART_REFERENCE_PARAM_IN", "")


@pytest.mark.skipif(not (SHIPPED and os.path.exists(SHIPPED)),
                    reason="GAZPART_REFERENCE_PARAM_IN does not name the reference's param.in")
def test_shipped_param_in():
    with pytest.raises(params.ParamError) as e:
        params.read_param(SHIPPED)
    assert e.value.line == 29
    p = params.read_param(SHIPPED, layout="file")
    assert (p.nx, p.ny, p.nz, p.dtime_user, p.ncyclemax) == (64, 64, 64, 1.0e-5, 10000)
    assert (p.nig, p.npart_full, p.interp_scheme, p.frozen_flow) == (1, 10000, 3, 1)
    assert (p.lxmax, p.visc, p.rhof) == (0.314, 1.515e-5, 1.205)
    c = p.classes[0]
    assert (c.partdef, c.collidef, c.emaj_part_user, c.apr_part, c.rhop_user) == (2, 1, 500.0e-6, 1.5, 1038.0)
    assert (p.ecw, p.muw, p.filtering, p.kcut) == (1.0, 0.0, False, 128.0)
