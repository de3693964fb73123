"""Reader/writer for the ``.LBMBin`` field files and the block-tiled node order.

Format (reference ``src/fileIO/fileOutput.cuh:82-183``): an ASCII header of
three blocks ``systemInformation{binaryType littleEndian; scalarType 32 bit;}``,
``fieldInformation{timeStep t; timeType instantaneous|timeAverage;
fieldNames[n]{...};}`` and ``fieldData{fieldType nonUniform;
field[N*n][n][nz][ny][nx] {`` followed by the raw little-endian values, a
newline and the closing ``};`` lines.  Values are ordered ``[field][node]``
with the node index in the reference's block-tiled order
``tx + 8*(ty + 8*(tz + 8*(bx + NBX*(by + NBY*bz))))`` (reference
``src/globalFunctions.cuh:208-214``, ``src/memory/memory.cuh:157-195``).

The product's writer is C++ (``cudalbm_b200/csrc/lbmbin.cpp``); this module is
for tests and tooling.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

BLOCK = 8


def block_tiled_index(nx: int, ny: int, nz: int) -> np.ndarray:
    """``idx[z, y, x]`` = position of node (x, y, z) in block-tiled order."""
    if nx % BLOCK or ny % BLOCK or nz % BLOCK:
        raise ValueError("mesh dimensions must be multiples of 8")
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    tx, ty, tz = x % BLOCK, y % BLOCK, z % BLOCK
    bx, by, bz = x // BLOCK, y // BLOCK, z // BLOCK
    nbx, nby = nx // BLOCK, ny // BLOCK
    return (tx + BLOCK * (ty + BLOCK * (tz + BLOCK * (bx + nbx * (by + nby * bz))))).astype(np.int64)


def tiled_to_global(data: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """Block-tiled flat array(s) ``[..., N]`` -> ``[..., nz, ny, nx]``."""
    idx = block_tiled_index(nx, ny, nz)
    return data[..., idx]


def global_to_tiled(data: np.ndarray) -> np.ndarray:
    """``[..., nz, ny, nx]`` -> block-tiled flat ``[..., N]``."""
    nz, ny, nx = data.shape[-3:]
    idx = block_tiled_index(nx, ny, nz).reshape(-1)
    out = np.empty(data.shape[:-3] + (nx * ny * nz,), dtype=data.dtype)
    out[..., idx] = data.reshape(data.shape[:-3] + (-1,))
    return out


@dataclass
class FieldFile:
    time_step: int
    time_type: str
    names: List[str]
    nx: int
    ny: int
    nz: int
    data: np.ndarray  # [nvars, nz, ny, nx] in global order

    def field(self, name: str) -> np.ndarray:
        return self.data[self.names.index(name)]


def read(path: str) -> FieldFile:
    with open(path, "rb") as fh:
        raw = fh.read()
    pos = 0
    names: List[str] = []
    time_step = None
    time_type = None
    scalar = None
    little = None
    dims = None
    in_names = False
    while pos < len(raw):
        end = raw.index(b"\n", pos)
        line = raw[pos:end].decode("ascii").strip()
        pos = end + 1
        if not line:
            continue
        if line.startswith("binaryType"):
            little = "littleEndian" in line
        elif line.startswith("scalarType"):
            scalar = 4 if "32 bit" in line else 8 if "64 bit" in line else None
        elif line.startswith("timeStep"):
            time_step = int(line.split()[1].rstrip(";"))
        elif line.startswith("timeType"):
            time_type = line.split()[1].rstrip(";")
        elif line.startswith("fieldNames["):
            in_names = True
        elif in_names:
            if line == "{":
                continue
            if line == "};":
                in_names = False
                continue
            names.append(line.rstrip(";"))
        elif line.startswith("field["):
            dims = [int(t.rstrip("]")) for t in line[len("field["):].split("[")]
            # the next non-empty line is "{", then binary data starts
            end = raw.index(b"\n", pos)
            if raw[pos:end].decode("ascii").strip() != "{":
                raise ValueError("malformed fieldData block")
            pos = end + 1
            break
    if dims is None or scalar is None or little is None:
        raise ValueError(f"{path}: incomplete header")
    total, nvars, nz, ny, nx = dims[:5]
    if total != nvars * nx * ny * nz or nvars != len(names):
        raise ValueError(f"{path}: inconsistent header dimensions")
    dtype = np.dtype(("<" if little else ">") + ("f4" if scalar == 4 else "f8"))
    nbytes = total * dtype.itemsize
    if pos + nbytes > len(raw):
        raise ValueError(f"{path}: truncated data ({len(raw) - pos} of {nbytes} bytes)")
    flat = np.frombuffer(raw, dtype=dtype, count=total, offset=pos).reshape(nvars, -1)
    data = tiled_to_global(flat, nx, ny, nz)
    return FieldFile(time_step, time_type, names, nx, ny, nz, np.ascontiguousarray(data))


def write(path: str, names: Sequence[str], data: np.ndarray, time_step: int,
          time_type: str = "instantaneous") -> None:
    """Write ``data[nvars, nz, ny, nx]`` (float32 or float64) as .LBMBin."""
    data = np.asarray(data)
    if data.dtype not in (np.float32, np.float64):
        raise TypeError("LBMBin fields are float32 or float64")
    nvars, nz, ny, nx = data.shape
    flat = global_to_tiled(data).astype(data.dtype.newbyteorder("<"), copy=False)
    bits = 32 if data.dtype.itemsize == 4 else 64
    hdr = ["systemInformation", "{", "\tbinaryType\tlittleEndian;", "", f"\tscalarType\t{bits} bit;", "};", "",
           "fieldInformation", "{", f"\ttimeStep\t{int(time_step)};", "", f"\ttimeType\t{time_type};", "",
           f"\tfieldNames[{nvars}]", "\t{"]
    hdr += [f"\t\t{n};" for n in names]
    hdr += ["\t};", "};", "", "fieldData", "{", "\tfieldType\tnonUniform;", "",
            f"\tfield[{nvars * nx * ny * nz}][{nvars}][{nz}][{ny}][{nx}]", "\t{"]
    with open(path, "wb") as fh:
        fh.write(("\n".join(hdr) + "\n").encode("ascii"))
        fh.write(flat.tobytes())
        fh.write(b"\n\t};\n};\n")
