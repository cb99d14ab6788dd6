"""Readers/writers for the reference-driver files (test infrastructure).

``read_records`` parses the record stream that oracle/ref_driver.cu writes:
{char name[64]; uint32 dtype (0 f32, 1 u32, 2 f64, 3 u64); uint64 count; data}.
``write_case`` writes the harness's plain-text case description.
"""
from __future__ import annotations

import struct
from typing import Dict, Iterable, Tuple

import numpy as np

_DT = {0: np.float32, 1: np.uint32, 2: np.float64, 3: np.uint64}


def read_records(path: str) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        name = data[pos:pos + 64].split(b"\0", 1)[0].decode()
        dtype, count = struct.unpack_from("<IQ", data, pos + 64)
        pos += 76
        dt = np.dtype(_DT[dtype])
        n = count * dt.itemsize
        out[name] = np.frombuffer(data[pos:pos + n], dtype=dt).copy()
        pos += n
    return out


def write_case(path: str, init: Tuple[float, float, float, float, float],
               bcs: Iterable[Tuple], cfl: float = 0.8, iters: int = 100, tol: float = 0.0,
               state: str | None = None) -> None:
    """bcs: ("slip", region) or ("farfield", region, mx, my, mz, p, T), applied in order."""
    lines = ["init %.9g %.9g %.9g %.9g %.9g" % tuple(init)]
    for b in bcs:
        if b[0] == "slip":
            lines.append(f"slip {b[1]}")
        else:
            lines.append("farfield %s %.9g %.9g %.9g %.9g %.9g" % tuple(b[1:]))
    lines += [f"cfl {cfl:.9g}", f"iters {iters}", f"tol {tol:.9g}"]
    if state:
        lines.append(f"state {state}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
