"""The reference's binary output layout, reused for initial conditions,
parity dumps and checkpoints.

``out%04d.dat``: one double (simulation time) followed by the state ``uu`` as
NVAR*nx*ny doubles in C order ``[NVAR][nx][ny]`` (``writeOutput.c:47-76``;
reader ``data_proc_scripts/read_output.py:40-46``).  ``xgrid.dat`` /
``ygrid.dat``: a ``size_t`` count followed by that many doubles
(``writeOutput.c:5-45``).  ``divB%04d.dat``: time then ``[nx][ny]`` doubles
(``writeOutput.c:78-107``).

A restart from such a file at a step boundary is exact: the only other
persistent array, ``dudtRK``, is zeroed by every ``rkInit`` (``timeAdvance.c:26``).
"""
from __future__ import annotations

import numpy as np


def write_state(path: str, uu: np.ndarray, t: float = 0.0) -> None:
    uu = np.ascontiguousarray(uu, dtype=np.float64)
    with open(path, "wb") as f:
        np.array([t], dtype=np.float64).tofile(f)
        uu.tofile(f)


def read_state(path: str, nvar: int, nx: int, ny: int):
    a = np.fromfile(path, dtype=np.float64)
    if a.size != 1 + nvar * nx * ny:
        raise ValueError(f"{path}: expected {1 + nvar * nx * ny} doubles, found {a.size}")
    return float(a[0]), a[1:].reshape(nvar, nx, ny)


def write_grid(path: str, coords: np.ndarray) -> None:
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    with open(path, "wb") as f:
        np.array([coords.size], dtype=np.uint64).tofile(f)
        coords.tofile(f)


def read_grid(path: str) -> np.ndarray:
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], dtype=np.uint64)[0])
    return np.frombuffer(raw[8:8 + 8 * n], dtype=np.float64).copy()


def write_divb(path: str, divb: np.ndarray, t: float = 0.0) -> None:
    write_state(path, divb.reshape(1, *divb.shape[-2:]), t)
