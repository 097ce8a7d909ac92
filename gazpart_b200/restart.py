"""The reference's particle restart and snapshot files (host side of ``gazpart_files.h``).

Two layouts, both Fortran sequential unformatted files read and written by the native
library (gfortran record markers, see ``include/gazpart_files.h``):

* the class restart of SAVE_PARTICLE with ISAVEPART = 2 (save_particle.f90:116-180),
  read back at start-up by INITIATION_PARTICLE_POSITION
  (initiation_particle_position.f90:430-532): a header with NPART_FULL and the class's
  polydisperse tables, then 14 columns;
* the snapshot of PRINT_PARTICLE (print_particle.f90:145-170): the 14 columns alone.

The 14 columns are x y z u v w, the quaternion a b c d, omega x y z and real(IDP), the
polydisperse index of each particle.  A third layout, the multi-class ``PART`` file of
ISAVEPART = 1, is written and read here with the generic record calls
(``write_part_multi``, ``read_part_multi``); the reference's reader for it expects
records its writer does not write, and this module reproduces both sides as they are.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check
from .api import PROP_KEYS, STATE_KEYS

PART_COLUMNS = STATE_KEYS + ("idp",)
NPARTCOL = 14
MAX_SUBRECORD = 2147483639


@dataclasses.dataclass
class ClassTables:
    """NPCLASS(J,:), RHOP(J,:), EMAJ_PART(J,:) and APR_PART(J) of one class."""
    npclass: np.ndarray
    rhop: np.ndarray
    emaj: np.ndarray
    apr: float

    def __post_init__(self):
        self.npclass = np.ascontiguousarray(self.npclass, dtype=np.int32)
        self.rhop = np.ascontiguousarray(self.rhop, dtype=np.float64)
        self.emaj = np.ascontiguousarray(self.emaj, dtype=np.float64)
        self.apr = float(self.apr)
        if not (self.npclass.size == self.rhop.size == self.emaj.size >= 1):
            raise ValueError("the three tables must have the same length >= 1")

    @property
    def polydisp(self) -> int:
        return int(self.npclass.size)


def default_tables(npart_full: int, emaj_user: float, apr: float, rhop_user: float, polydisp: int = 1,
                   polydispmax: Optional[int] = None, partdef: int = 2, nq_np: float = 0.0,
                   rhoq_rhop: float = 1.0, idp: Optional[np.ndarray] = None) -> ClassTables:
    """The tables a fresh run holds for one class.

    Defaults RHOP = RHOP_USER, EMAJ_PART = EMAJ_PART_USER and NPCLASS = NPART_FULL over
    all POLYDISPMAX entries (init_run.f90:318-341).  A bidisperse inertial class takes
    RHOP(J,2) = RHOP_USER/RHOQ_RHOP (initiation_particle_position.f90:176-215).  When
    POLYDISP > 1 the entries 1..POLYDISP of NPCLASS count the particles of each index
    (initiation_particle_position.f90:583-595); give idp for that, otherwise the
    reference's own split int(N/(1+NQ_NP)) of index 1 then index 2 is counted."""
    pdm = polydisp if polydispmax is None else polydispmax
    rhop = np.full(pdm, float(rhop_user))
    emaj = np.full(pdm, float(emaj_user))
    npclass = np.full(pdm, int(npart_full), dtype=np.int32)
    if polydisp > 1:
        if partdef >= 2:
            rhop[1] = float(rhop_user) / float(rhoq_rhop)
        if idp is None:
            idp = initial_idp(npart_full, polydisp, nq_np)
        counts = np.bincount(np.asarray(idp, dtype=np.int64) - 1, minlength=polydisp)[:polydisp]
        npclass[:polydisp] = counts
    return ClassTables(npclass=npclass, rhop=rhop, emaj=emaj, apr=apr)


def initial_idp(n: int, polydisp: int, nq_np: float = 0.0) -> np.ndarray:
    """IDP of a fresh class: 1 throughout, or for POLYDISP > 1 index 1 for the first
    int(N/(1+NQ_NP)) particles and 2 for the rest (initiation_particle_position.f90:178-185)."""
    idp = np.ones(n, dtype=np.int32)
    if polydisp > 1:
        idp[int(n / (1.0 + nq_np)):] = 2
    return idp


def props_from_tables(idp: np.ndarray, tables: ClassTables) -> Dict[str, np.ndarray]:
    """Per-particle constants from the class tables: EMAJ_PART(J,IDP), APR_PART(J),
    RHOP(J,IDP) and the inertia of initiation_particle_position.f90:609-624."""
    k = np.asarray(idp, dtype=np.int64) - 1
    if k.size and (k.min() < 0 or k.max() >= tables.polydisp):
        raise ValueError("IDP outside 1..POLYDISP")
    a = tables.emaj[k]
    b = a / tables.apr
    c = b
    return {"emaj": a, "apr": np.full(k.size, tables.apr), "rhop": tables.rhop[k],
            "ipxx": (b * b + c * c) / 5.0, "ipyy": (a * a + c * c) / 5.0, "ipzz": (a * a + b * b) / 5.0}


def _fortran_int(v: int, w: int) -> str:
    """Iw.w edit descriptor: at least w digits, w asterisks when it does not fit."""
    s = f"{abs(v):0{w}d}"
    if v < 0:
        s = "-" + s
    return "*" * w if len(s) > w else s


def part_file_name(j: int, ncycle: Optional[int] = None, kind: str = "bin") -> str:
    """File names of the class restart: part_pJJ_tNNNNNNNN.bin for a cycle,
    part_pJJ.end for the final state (save_particle.f90:148-152, formats 10100 and
    10102), and part_pJJ.ini for the file a run starts from
    (initiation_particle_position.f90:440)."""
    if kind == "bin":
        if ncycle is None or ncycle < 0:
            raise ValueError("a .bin name needs a cycle number >= 0")
        return f"part_p{_fortran_int(j, 2)}_t{_fortran_int(ncycle, 8)}.bin"
    if kind in ("end", "ini"):
        return f"part_p{_fortran_int(j, 2)}.{kind}"
    raise ValueError("kind must be 'bin', 'end' or 'ini'")


def snapshot_file_name(j: int, ncycle: int) -> str:
    """PRINT_PARTICLE's postprocessing/part_pJJ_tNNNNNNNN.bin (print_particle.f90:147)."""
    return "postprocessing/" + part_file_name(j, ncycle, "bin")


def _b(path: str) -> bytes:
    return os.fsencode(path)


def _col_ptrs(cols: Sequence[np.ndarray]):
    return (C.c_void_p * len(cols))(*[C.c_void_p(c.ctypes.data) for c in cols])


class FortranFile:
    """A sequential unformatted file: write() is one WRITE, read() one READ."""

    def __init__(self, path: str, mode: str = "r", max_subrecord: Optional[int] = None):
        if mode not in ("r", "w"):
            raise ValueError("mode must be 'r' or 'w'")
        self._h = C.c_void_p()
        check(_lib.lib().gp_funf_open(_b(path), 1 if mode == "w" else 0, C.byref(self._h)), "gp_funf_open")
        if max_subrecord is not None:
            check(_lib.lib().gp_funf_set_max_subrecord(self._h, int(max_subrecord)), "gp_funf_set_max_subrecord")

    def write(self, *arrays) -> None:
        """One record holding the arrays back to back."""
        data = b"".join(np.ascontiguousarray(a).tobytes() for a in arrays) if len(arrays) != 1 else None
        if data is None:
            a = np.ascontiguousarray(arrays[0])
            check(_lib.lib().gp_funf_write(self._h, C.c_void_p(a.ctypes.data), a.nbytes), "gp_funf_write")
        else:
            buf = C.create_string_buffer(data, len(data))
            check(_lib.lib().gp_funf_write(self._h, C.cast(buf, C.c_void_p), len(data)), "gp_funf_write")

    def record_size(self) -> int:
        n = C.c_int64()
        check(_lib.lib().gp_funf_record_size(self._h, C.byref(n)), "gp_funf_record_size")
        return n.value

    def read(self, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype=dtype)
        check(_lib.lib().gp_funf_read(self._h, C.c_void_p(out.ctypes.data) if count else None, out.nbytes),
              "gp_funf_read")
        return out

    def read_record(self, dtype) -> np.ndarray:
        """The whole next record as an array of dtype."""
        n = self.record_size()
        return self.read(dtype, n // np.dtype(dtype).itemsize)

    def skip(self) -> None:
        check(_lib.lib().gp_funf_read(self._h, None, 0), "gp_funf_read")

    def close(self) -> None:
        if self._h:
            h, self._h = self._h, C.c_void_p()
            check(_lib.lib().gp_funf_close(h), "gp_funf_close")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _columns(cols: Dict[str, np.ndarray], n: Optional[int] = None) -> List[np.ndarray]:
    out = []
    for k in PART_COLUMNS:
        a = np.ascontiguousarray(np.asarray(cols[k], dtype=np.float64))
        if n is None:
            n = a.size
        if a.size != n:
            raise ValueError(f"column {k} has {a.size} values, not {n}")
        out.append(a)
    return out


def write_part_class(path: str, cols: Dict[str, np.ndarray], tables: ClassTables) -> None:
    """SAVE_PARTICLE's class restart file (ISAVEPART = 2).  cols: the 13 state columns
    and "idp" (written as real(IDP))."""
    arr = _columns(cols)
    n = arr[0].size
    check(_lib.lib().gp_write_part_class(_b(path), n, tables.polydisp,
                                         tables.npclass.ctypes.data_as(_lib._ip),
                                         tables.rhop.ctypes.data_as(_lib._dp),
                                         tables.emaj.ctypes.data_as(_lib._dp), tables.apr, _col_ptrs(arr)),
          "gp_write_part_class")


def read_part_class(path: str) -> Tuple[Dict[str, np.ndarray], ClassTables]:
    """What INITIATION_PARTICLE_POSITION reads from a class restart file: the 14 columns
    (IDP as the reference's int(column 14)) and the tables."""
    n, pd = C.c_int64(), C.c_int32()
    check(_lib.lib().gp_read_part_class_header(_b(path), C.byref(n), C.byref(pd)), "gp_read_part_class_header")
    n, pd = n.value, pd.value
    npclass = np.empty(pd, np.int32)
    rhop, emaj = np.empty(pd), np.empty(pd)
    apr = C.c_double()
    arr = [np.empty(n) for _ in range(NPARTCOL)]
    check(_lib.lib().gp_read_part_class(_b(path), n, pd, npclass.ctypes.data_as(_lib._ip),
                                        rhop.ctypes.data_as(_lib._dp), emaj.ctypes.data_as(_lib._dp),
                                        C.byref(apr), _col_ptrs(arr)), "gp_read_part_class")
    cols = dict(zip(PART_COLUMNS, arr))
    cols["idp"] = np.trunc(cols["idp"]).astype(np.int32)
    return cols, ClassTables(npclass=npclass, rhop=rhop, emaj=emaj, apr=apr.value)


def write_snapshot(path: str, cols: Dict[str, np.ndarray]) -> None:
    """PRINT_PARTICLE's snapshot: the 14 columns, no header."""
    arr = _columns(cols)
    check(_lib.lib().gp_write_part_snapshot(_b(path), arr[0].size, _col_ptrs(arr)), "gp_write_part_snapshot")


def read_snapshot(path: str) -> Dict[str, np.ndarray]:
    with FortranFile(path) as f:
        n = f.record_size() // 8
    arr = [np.empty(n) for _ in range(NPARTCOL)]
    check(_lib.lib().gp_read_part_snapshot(_b(path), n, _col_ptrs(arr)), "gp_read_part_snapshot")
    cols = dict(zip(PART_COLUMNS, arr))
    cols["idp"] = np.trunc(cols["idp"]).astype(np.int32)
    return cols


def upload_dict(cols: Dict[str, np.ndarray], tables: ClassTables) -> Dict[str, np.ndarray]:
    """A restart file's columns as the state and constants Context.upload takes."""
    out = {k: np.ascontiguousarray(cols[k], dtype=np.float64) for k in STATE_KEYS}
    out.update(props_from_tables(cols["idp"], tables))
    return out


def save_class(ctx, ig: int, path: str, tables: ClassTables, idp: Optional[np.ndarray] = None) -> None:
    """Class ig of a context into a class restart file, straight from the device
    (gp_save_part_class).  idp: each particle's polydisperse index, or all 1."""
    ip = None
    if idp is not None:
        idp = np.ascontiguousarray(idp, dtype=np.int32)
        ip = idp.ctypes.data_as(_lib._ip)
    check(_lib.lib().gp_save_part_class(ctx._h, int(ig), _b(path), tables.polydisp,
                                        tables.npclass.ctypes.data_as(_lib._ip),
                                        tables.rhop.ctypes.data_as(_lib._dp),
                                        tables.emaj.ctypes.data_as(_lib._dp), tables.apr, ip),
          "gp_save_part_class")


def load_class(ctx, path: str, field: int = 0) -> Tuple[int, int]:
    """A class restart file into a context as a new class (gp_load_part_class); returns
    (class number, particles)."""
    ig, n = C.c_int32(), C.c_int64()
    check(_lib.lib().gp_load_part_class(ctx._h, _b(path), int(field), C.byref(ig), C.byref(n)),
          "gp_load_part_class")
    ctx.n += n.value
    return ig.value, n.value


# ISAVEPART = 1: one file for all classes
_MULTI_WRITTEN = ("x", "y", "z", "u", "v", "w", "ufap", "vfap", "wfap")
_MULTI_READ = ("dummy", "x", "y", "z", "u", "v", "w", "ufap", "vfap", "wfap",
               "qa", "qb", "qc", "qd", "ox", "oy", "oz")


def write_part_multi(path: str, classes: Sequence[Dict[str, np.ndarray]]) -> None:
    """SAVE_PARTICLE with ISAVEPART = 1 (save_particle.f90:73-96): per class NPART_LOC,
    IDP (int32), then x y z u v w and the fluid velocity seen ufap vfap wfap."""
    with FortranFile(path, "w") as f:
        for c in classes:
            n = int(np.asarray(c["x"]).size)
            f.write(np.array([n], np.int32))
            f.write(np.asarray(c["idp"], np.int32))
            for k in _MULTI_WRITTEN:
                f.write(np.asarray(c[k], np.float64))


def read_part_multi(path: str, nig: int, npmax_loc: Optional[int] = None) -> List[Dict[str, np.ndarray]]:
    """INITIATION_PARTICLE_POSITION with ISAVEPART = 1
    (initiation_particle_position.f90:360-424): per class NP_READ, IDP, one record of
    NP_READ reals it discards, x y z u v w, ufap vfap wfap, the quaternion and omega.
    On a file of write_part_multi this fails as the reference does: the discarded read
    takes the x record, and the last reads of the class run past the end of a record
    (GP_ERECORD) or of the file (GP_EEOF)."""
    out = []
    with FortranFile(path) as f:
        for _ in range(nig):
            n = int(f.read(np.int32, 1)[0])
            if npmax_loc is not None and n > npmax_loc:
                raise ValueError(f"NP_READ={n} > NPMAX_LOC={npmax_loc}")
            c = {"idp": f.read(np.int32, n)}
            for k in _MULTI_READ:
                c[k] = f.read(np.float64, n)
            del c["dummy"]
            out.append(c)
    return out
