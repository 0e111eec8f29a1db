"""Run parameters in the reference's ``input`` layout.

The reference reads a 15-line text file ``input`` and keeps only the first
16 characters of every line, which it converts with ``atoi``/``atof``
(``initialize.c:442-525``; line order in the shipped ``input:1-15``).  This
module writes and reads that layout with the same 16-character rule, so the
GPU path and the reference see bit-identical parameters (``Lx = 2*pi``, for
instance, is 16 significant characters, not a full double).

Derived quantities follow ``initialize.c:123-154``: ``dx = Lx/nx`` for a
periodic x boundary (``Lx/(nx-1)`` for open), ``dy = Ly/ny``,
``constDiffDivB = 2 * max(dx, dy)**2``, ``NVAR = 9`` with hyperbolic divergence
cleaning (``divBcleaning == 2``) and 8 otherwise (``initialize.c:207-214``).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import re

# order of the 15 lines (initialize.c:465-522)
FIELDS = (
    ("boundaryTypeX", int),
    ("cfl", float),
    ("Tmax", float),
    ("dtOut", float),
    ("nx", int),
    ("ny", int),
    ("Lx", float),
    ("Ly", float),
    ("adiabaticIdx", float),
    ("Hall", int),
    ("di", float),
    ("resistivity", float),
    ("viscosity", float),
    ("divBcleaning", int),
    ("outDivB", int),
)

_INT_RE = re.compile(r"^\s*([+-]?\d+)")
_FLT_RE = re.compile(r"^\s*([+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)")


def _atoi(s: str) -> int:
    m = _INT_RE.match(s)
    return int(m.group(1)) if m else 0


def _atof(s: str) -> float:
    m = _FLT_RE.match(s)
    return float(m.group(1)) if m else 0.0


def _fmt16(v) -> str:
    """Shortest text of ``v`` that fits in 16 characters (the reference keeps
    only 16 characters per line)."""
    if isinstance(v, int):
        s = str(v)
    else:
        s = repr(float(v))
        if len(s) > 16:
            for prec in range(16, 0, -1):
                s = f"{float(v):.{prec}g}"
                if len(s) <= 16:
                    break
    if len(s) > 16:
        raise ValueError(f"value {v!r} does not fit the 16-character input field")
    return s


@dataclasses.dataclass
class InputParams:
    """The 15 run parameters of the reference's ``input`` file."""

    boundaryTypeX: int = 0
    cfl: float = 0.3
    Tmax: float = 1.0
    dtOut: float = 0.1
    nx: int = 256
    ny: int = 256
    Lx: float = 2 * math.pi
    Ly: float = 2 * math.pi
    adiabaticIdx: float = 5.0 / 3.0
    Hall: int = 0
    di: float = 0.0
    resistivity: float = 1e-4
    viscosity: float = 1e-4
    divBcleaning: int = 0
    outDivB: int = 0

    # -- the reference's text layout -------------------------------------
    def to_text(self) -> str:
        out = []
        for name, _ in FIELDS:
            v = getattr(self, name)
            out.append(f"{_fmt16(v):<20s}; {name}\n")
        return "".join(out)

    def write(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.to_text())

    @classmethod
    def from_text(cls, text: str) -> "InputParams":
        lines = text.splitlines()
        if len(lines) < len(FIELDS):
            raise ValueError("input needs 15 lines")
        kw = {}
        for (name, typ), line in zip(FIELDS, lines):
            head = line[:16]
            kw[name] = _atoi(head) if typ is int else _atof(head)
        return cls(**kw)

    @classmethod
    def read(cls, path: str) -> "InputParams":
        with open(path) as f:
            return cls.from_text(f.read())

    def normalized(self) -> "InputParams":
        """The values the reference would see after its 16-character parse."""
        return InputParams.from_text(self.to_text())

    # -- derived quantities (initialize.c:123-154, 207-214) --------------
    @property
    def nvar(self) -> int:
        return 9 if self.divBcleaning == 2 else 8

    @property
    def dx(self) -> float:
        return self.Lx / self.nx if self.boundaryTypeX == 0 else self.Lx / (self.nx - 1)

    @property
    def dy(self) -> float:
        return self.Ly / self.ny

    @property
    def const_diff_divb(self) -> float:
        m = max(self.dx, self.dy)
        return 2.0 * m * m

    def state_shape(self) -> tuple:
        return (self.nvar, self.nx, self.ny)


class CParams(ctypes.Structure):
    """C mirror of ``mhdgpu_params`` (include/mhd_gpu.h)."""

    _fields_ = [
        ("boundaryTypeX", ctypes.c_int),
        ("cfl", ctypes.c_double),
        ("Tmax", ctypes.c_double),
        ("dtOut", ctypes.c_double),
        ("nx", ctypes.c_long),
        ("ny", ctypes.c_long),
        ("Lx", ctypes.c_double),
        ("Ly", ctypes.c_double),
        ("adiabaticIdx", ctypes.c_double),
        ("Hall", ctypes.c_int),
        ("di", ctypes.c_double),
        ("resistivity", ctypes.c_double),
        ("viscosity", ctypes.c_double),
        ("divBcleaning", ctypes.c_int),
        ("outDivB", ctypes.c_int),
    ]

    @classmethod
    def from_params(cls, p: InputParams) -> "CParams":
        return cls(**{name: getattr(p, name) for name, _ in FIELDS})
