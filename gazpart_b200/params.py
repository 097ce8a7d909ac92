"""The reference's ``param.in`` importer: READPARAM (readparam.f90:1-277) restated.

READPARAM reads ``param.in`` with one list-directed READ per line, in a fixed order,
into module variables.  This module reads the same statements in the same order with
Fortran list-directed semantics:

* a READ with no items passes over one record;
* values are separated by blanks or commas, a slash ends the READ and leaves the rest
  of its items unchanged, ``r*c`` repeats a value and ``r*`` gives r null values;
* a READ that wants more values than its record holds continues on the next record,
  and what is left of the last record it used is passed over;
* '!' is not a comment character: it only ends a READ when all its items are filled
  before it, so text after the wanted values is never looked at;
* a logical is an optional '.', then T or F, then anything up to a separator; an
  integer is an optional sign and digits; a real takes an optional exponent with E, D
  or Q, or a bare signed exponent.  A value of the wrong form is an error, as it is in
  the compiled reader ('Bad integer for item 1 in list input').

The reader and the ``param.in`` shipped beside it disagree: the file has a
``DRY_CHANNEL`` line after ``SOLVE_PART`` that the reader no longer reads
(readparam.f90:75, commented out), so READPARAM stops on it, reading ``.false.`` as
the integer ``NIG``.  ``read_param(..., layout="reader")`` does exactly that.
``layout="file"`` also reads the ``DRY_CHANNEL`` record, which is what the shipped file
needs.

After the reads, READPARAM's own adjustments follow (readparam.f90:240-277): a class
whose PARTDEF is below 2 gets COLLIDEF = 0, SOLVE_COLLISION is set when any class
collides, PERIODICITY = not WALL_BOUNDARY, FOUT1..3 are capped at NCYCLEMAX, and more
than 20 classes are refused.
"""
from __future__ import annotations

import dataclasses
import re
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import config


class ParamError(ValueError):
    """A READ that the compiled reader would stop on (line numbers are 1-based)."""

    def __init__(self, message: str, line: int):
        self.line = line
        super().__init__(f"param.in line {line}: {message}")


_INT = re.compile(r"[+-]?\d+\Z")
_REAL = re.compile(r"([+-]?(?:\d+\.?\d*|\.\d+))(?:([EeDdQq])([+-]?\d+)|([+-]\d+))?\Z")


def _logical(tok: str) -> Optional[bool]:
    t = tok[1:] if tok.startswith(".") else tok
    if t[:1] in ("T", "t"):
        return True
    if t[:1] in ("F", "f"):
        return False
    return None


def _convert(tok: str, kind: str, item: int, line: int):
    if kind == "i":
        if not _INT.match(tok):
            raise ParamError(f"Bad integer for item {item} in list input ({tok!r})", line)
        return int(tok)
    if kind == "l":
        v = _logical(tok)
        if v is None:
            raise ParamError(f"Bad logical value for item {item} in list input ({tok!r})", line)
        return v
    m = _REAL.match(tok)
    if not m:
        raise ParamError(f"Bad real number in item {item} of list input ({tok!r})", line)
    mant, _, e1, e2 = m.groups()
    exp = e1 if e1 is not None else e2
    return float(mant + ("e" + exp if exp is not None else ""))


class _ListReader:
    """Fortran list-directed READs over the lines of a file."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0          # index of the next record

    def _tokens(self, rec: str) -> List[Optional[str]]:
        """Values of one record: strings, None for a null value, '/' for a slash."""
        out: List[Optional[str]] = []
        i, n = 0, len(rec)
        last_comma = True     # a comma right at the start, or after a comma, is a null
        while i < n:
            c = rec[i]
            if c in " \t":
                i += 1
                continue
            if c == ",":
                if last_comma:
                    out.append(None)
                last_comma = True
                i += 1
                continue
            if c == "/":
                out.append("/")
                return out
            j = i
            while j < n and rec[j] not in " \t,/":
                j += 1
            tok = rec[i:j]
            m = re.match(r"(\d+)\*(.*)\Z", tok)
            if m:
                r = int(m.group(1))
                out.extend([m.group(2) or None] * r)
            else:
                out.append(tok)
            last_comma = False
            i = j
            # a following comma belongs to this value
            while i < n and rec[i] in " \t":
                i += 1
            if i < n and rec[i] == ",":
                i += 1
                last_comma = True
        return out

    def read(self, kinds: Sequence[str]) -> List[Optional[object]]:
        """One READ statement.  kinds: 'i', 'r' or 'l' per item; None for items left
        unchanged (null values or a slash)."""
        vals: List[Optional[object]] = [None] * len(kinds)
        if self.pos >= len(self.lines):
            raise ParamError("End of file", self.pos + 1)
        if not kinds:
            self.pos += 1
            return vals
        k = 0
        while k < len(kinds):
            if self.pos >= len(self.lines):
                raise ParamError("End of file", self.pos + 1)
            line = self.pos + 1
            toks = self._tokens(self.lines[self.pos])
            self.pos += 1
            for tok in toks:
                if tok == "/":
                    return vals
                if tok is not None:
                    vals[k] = _convert(tok, kinds[k], k + 1, line)
                k += 1
                if k == len(kinds):
                    break
        return vals


@dataclasses.dataclass
class ParticleClass:
    """One class's block of READPARAM section 8 (readparam.f90:200-232)."""
    partdef: int
    collidef: int
    emaj_part_user: float
    apr_part: float
    rhop_user: float
    ecp: float
    mup: float
    gravity: float
    cp_part: float
    polydisp: int
    nq_np: float
    dq_dp: float
    rhoq_rhop: float


@dataclasses.dataclass
class Params:
    """The module variables READPARAM sets, under the reference's names (lower case)."""
    values: Dict[str, object]
    classes: List[ParticleClass]
    layout: str

    def __getattr__(self, name: str):
        v = self.__dict__.get("values", {})
        if name in v:
            return v[name]
        raise AttributeError(name)

    def setup(self, ig: int = 1) -> config.Setup:
        """The mesh and physics of class ig as this package's Setup.

        Only the paths this package implements are accepted: Lagrange cubic
        interpolation (INTERP_SCHEME = 3), inertial particles (PARTDEF = 2) and a frozen
        field (FROZEN_FLOW = 1, 2 or 3, the last the channel)."""
        if self.interp_scheme != 3:
            raise ValueError(f"INTERP_SCHEME = {self.interp_scheme}: only 3 (interp_lag3.f90) is implemented")
        c = self.classes[ig - 1]
        if c.partdef != 2:
            raise ValueError(f"class {ig}: PARTDEF = {c.partdef}: only inertial particles (2) are advanced")
        if self.frozen_flow not in (1, 2, 3):
            raise ValueError(f"FROZEN_FLOW = {self.frozen_flow}: only a frozen field (1, 2, 3) is advanced")
        return config.Setup(nx=self.nx, ny=self.ny, nz=self.nz, lx=self.lxmax, ly=self.lymax, lz=self.lzmax,
                            visc=self.visc, rhof=self.rhof, dtime=self.dtime_user, gravity=c.gravity,
                            ecp=c.ecp, mup=c.mup, ecw=self.ecw, muw=self.muw,
                            periodicity=self.periodicity, wall_boundary=self.wall_boundary,
                            frozen_flow=self.frozen_flow)

    def tables(self, ig: int = 1):
        """Class ig's polydisperse tables as a fresh run builds them before any particle
        is placed (init_run.f90:318-341, initiation_particle_position.f90:176-215)."""
        from .restart import default_tables
        c = self.classes[ig - 1]
        pdmax = max(k.polydisp for k in self.classes)
        return default_tables(self.npart_full, c.emaj_part_user, c.apr_part, c.rhop_user, polydisp=c.polydisp,
                              polydispmax=pdmax, partdef=c.partdef, nq_np=c.nq_np, rhoq_rhop=c.rhoq_rhop)


# READPARAM sections 1-7 in order: a name and kind per item, () for a comment READ
_HEAD: List[Tuple[Tuple[str, str], ...]] = (
    [()] * 4 + [()] * 3 +
    [(("solve_fluid", "i"),), (), (("nx", "i"),), (("ny", "i"),), (("nz", "i"),), (),
     (("dtime_user", "r"),), (("ncyclemax", "i"),)] +
    [(), (("frozen_flow", "i"),), (("init_fluid_velocity", "i"),), (("steady", "l"),),
     (("sigma_force", "r"),), (("time_force", "r"),), (("kforce_min", "r"),), (("kforce_max", "r"),)] +
    [(), (("solve_scalar", "l"),), (("init_scalar", "i"),)] +
    [(), (("solve_part", "l"),)])
_PART_NUMERICS = [(("nig", "i"),), (("npart_full", "i"),), (("wall_boundary", "l"),), (("interp_scheme", "i"),),
                  (("init_part_position", "i"),), (("init_part_velocity", "i"),), (("init_part_scalar", "i"),)]
_TAIL = (
    [()] * 3 + [(("readstat", "l"),), (("stat_time", "l"),), (), (("level_stflu", "i"),), (),
                (("level1_stscl", "l"),), (("level2_stscl", "l"),), (),
                (("level1_stpar", "l"),), (("level2_stpar", "l"),), (("level3_stpar", "l"),),
                (("levelx_stpar", "l"),), (("level1_stpdf", "l"),)] +
    [()] * 3 + [(("fout0", "i"),), (("fout1", "i"),), (("fout2", "i"),), (("fout3", "i"),), (("fout4", "i"),),
                (("fout5", "i"),), (("ensight_out", "i"),), (("nslice", "i"),), (("refine_mesh", "r"),)] +
    [()] * 3 + [(("lxmax", "r"),), (("lymax", "r"),), (("lzmax", "r"),), (("visc", "r"),), (("rhof", "r"),)] +
    [()] * 3 + [(("diff_scl", "r"),), (("cp_scl", "r"),), (("grad_scl", "r"),)] +
    [()] * 3)
_CLASS = [(("partdef", "i"), ("collidef", "i")), (("emaj_part_user", "r"),), (("apr_part", "r"),),
          (("rhop_user", "r"),), (("ecp", "r"), ("mup", "r")), (("gravity", "r"),), (("cp_part", "r"),),
          (("polydisp", "i"),), (("nq_np", "r"), ("dq_dp", "r"), ("rhoq_rhop", "r")), ()]
_WALL = [(("ecw", "r"),), (("muw", "r"),), (("betaw", "r"),), (), (("filtering", "l"), ("kcut", "r"))]


def _run(reader: _ListReader, stmts, into: Dict[str, object]) -> None:
    for items in stmts:
        vals = reader.read([k for _, k in items])
        for (name, _), v in zip(items, vals):
            if v is not None or name not in into:
                into[name] = v


def parse_param(text: str, layout: str = "reader") -> Params:
    """READPARAM on the text of a ``param.in``.  layout: "reader" reads exactly the
    statements of readparam.f90; "file" also reads the DRY_CHANNEL record that the
    shipped param.in carries after SOLVE_PART."""
    if layout not in ("reader", "file"):
        raise ValueError("layout must be 'reader' or 'file'")
    r = _ListReader(text)
    v: Dict[str, object] = {}
    _run(r, _HEAD, v)
    if layout == "file":
        _run(r, [(("dry_channel", "l"),)], v)
    _run(r, _PART_NUMERICS, v)
    _run(r, _TAIL, v)
    nig = v["nig"]
    if nig is None or nig < 1:
        raise ParamError(f"NIG = {nig}", r.pos)
    classes = []
    for _ in range(nig):
        c: Dict[str, object] = {}
        _run(r, _CLASS, c)
        if c["polydisp"] == 1:          # readparam.f90:224-228
            c["nq_np"], c["dq_dp"], c["rhoq_rhop"] = 0.0, 1.0, 1.0
        classes.append(ParticleClass(**c))
    _run(r, _WALL, v)
    # readparam.f90:240-277
    for c in classes:
        if c.partdef < 2:
            c.collidef = 0
    v["solve_collision"] = sum(c.collidef for c in classes) > 0
    v["periodicity"] = not v["wall_boundary"]
    for k in ("fout1", "fout2", "fout3"):
        if v[k] is not None and v["ncyclemax"] is not None and v[k] > v["ncyclemax"]:
            v[k] = v["ncyclemax"]
    if nig > 20:
        raise ParamError(f"NIG={nig} > 20", r.pos)
    return Params(values=v, classes=classes, layout=layout)


def read_param(path: str, layout: str = "reader") -> Params:
    with open(path) as f:
        return parse_param(f.read(), layout)


def format_param(p: Params) -> str:
    """A ``param.in`` in the reader's own layout ("reader") holding p's values: one
    value per line, in READPARAM's order, with a short label after '!'."""
    v = p.values
    lines: List[str] = []

    def fmt(x, kind):
        if kind == "l":
            return ".true." if x else ".false."
        if kind == "i":
            return str(int(x))
        return repr(float(x))

    def emit(stmts, src):
        for items in stmts:
            if not items:
                lines.append("!")
                continue
            lines.append("  ".join(fmt(src[n], k) for n, k in items) + "   ! " + ", ".join(n.upper() for n, _ in items))

    emit(_HEAD, v)
    if p.layout == "file":
        emit([(("dry_channel", "l"),)], {"dry_channel": v.get("dry_channel", False)})
    emit(_PART_NUMERICS, v)
    emit(_TAIL, v)
    for c in p.classes:
        emit(_CLASS, dataclasses.asdict(c))
    emit(_WALL, v)
    return "\n".join(lines) + "\n"
