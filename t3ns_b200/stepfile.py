"""Reader for step-description files (``*.t3c``).

A step file holds everything the effective-Hamiltonian matvec of one
optimisation step needs, exactly as the reference sweep driver hands it to
``init_Heffdata`` (reference ``include/Heff.h:54-155``): the multi-site tensor
structure, the symsecs of every bond, the two or three renormalised operator
sets with their block tables and elements, the merge instruction set
(``include/instructions.h:39-66``), plus the replay schedule the reference built
for that step (``struct secondrun``, ``include/Heff.h:36-51``) and reference
matvec / diagonal / Davidson outputs.

Layout: the 8-byte magic ``T3NSCAP1`` followed by records
``{char name[48]; int32 dtype; int32 pad; int64 count; payload}`` with dtype
1 = int32, 2 = int64, 3 = float64, little endian.  A dtype with bit 0x10 set
marks a zlib-compressed payload: an int64 byte length, then the compressed
bytes of the ``count`` elements (used for the large schedule arrays of
structure-only benchmark files).
"""
from __future__ import annotations

import zlib

import numpy as np

_DTYPES = {1: np.int32, 2: np.int64, 3: np.float64}
_HDR = np.dtype([("name", "S48"), ("dtype", "<i4"), ("pad", "<i4"), ("count", "<i8")])


def synthesize_operator_values(n: int, opset: int) -> np.ndarray:
    """Operator elements of a structure-only step file: N(0, 0.1^2) from the
    fixed seed 2024 + opset (numpy PCG64)."""
    return np.random.default_rng(2024 + opset).standard_normal(n) * 0.1


def read_step(path) -> dict:
    """Return ``{name: ndarray}`` for every record of a step file.  For a
    structure-only file (``ops{i}.tel_len`` instead of ``ops{i}.tel``) the
    operator elements are synthesized (``synthesize_operator_values``)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"T3NSCAP1":
        raise ValueError(f"{path}: not a step file")
    out = {}
    pos = 8
    while pos < len(buf):
        hdr = np.frombuffer(buf, _HDR, 1, pos)[0]
        pos += _HDR.itemsize
        code = int(hdr["dtype"])
        dt = np.dtype(_DTYPES[code & 0xF])
        n = int(hdr["count"])
        if code & 0x10:
            nb = int(np.frombuffer(buf, np.int64, 1, pos)[0])
            pos += 8
            arr = np.frombuffer(zlib.decompress(buf[pos:pos + nb]), dt, n).copy()
            pos += nb
        else:
            arr = np.frombuffer(buf, dt, n, pos).copy()
            pos += n * dt.itemsize
        out[hdr["name"].decode()] = arr
    for i in range(3):
        if f"ops{i}.tel_len" in out and f"ops{i}.tel" not in out:
            out[f"ops{i}.tel"] = synthesize_operator_values(int(out[f"ops{i}.tel_len"][0]), i)
    return out


def write_step(path, rec: dict, compress_above: int | None = None) -> None:
    """Write ``{name: ndarray}`` in the step-file layout (int32/int64/float64);
    arrays of more than ``compress_above`` bytes are written zlib-compressed
    (never, by default)."""
    codes = {np.dtype(np.int32): 1, np.dtype(np.int64): 2, np.dtype(np.float64): 3}
    with open(path, "wb") as f:
        f.write(b"T3NSCAP1")
        for name, arr in rec.items():
            arr = np.ascontiguousarray(arr)
            h = np.zeros(1, _HDR)
            h["name"] = name.encode()
            h["count"] = arr.size
            if compress_above is not None and arr.nbytes > compress_above:
                payload = zlib.compress(arr.tobytes(), 6)
                h["dtype"] = codes[arr.dtype] | 0x10
                f.write(h.tobytes())
                f.write(np.array([len(payload)], np.int64).tobytes())
                f.write(payload)
            else:
                h["dtype"] = codes[arr.dtype]
                f.write(h.tobytes())
                f.write(arr.tobytes())
