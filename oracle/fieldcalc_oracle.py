"""CPU restatement of fieldCalculate's containsNaN and spatialMean.

TEST INFRASTRUCTURE ONLY: imported by tests/ to check lbm_field_statistics
and the fieldCalculate executable; the product never imports it.

Follows applications/fieldCalculate/fieldCalculate.cuh:
  * containsNaN (lines 74-84): a field contains NaN if any value is NaN
    (std::isnan; infinities are not NaN); the per-time block (lines 92-122)
    names each such field and counts them;
  * spatialMean (lines 130-140): ``sum += value`` in float over the field in
    global node order (x fastest; fileInput.cuh:777-820 de-interleaves the
    block-tiled file into that order), then ``sum / float(size)``; the block
    (lines 148-167) prints it with the stream's default 6 significant digits.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def spatial_mean(field_global: np.ndarray) -> np.float32:
    """Left-to-right float32 sum (numpy's accumulate is sequential) / float32(n)."""
    f = np.ascontiguousarray(field_global, dtype=np.float32).ravel()
    if f.size == 0:
        return np.float32(np.nan)
    s = np.add.accumulate(f, dtype=np.float32)[-1]
    return np.float32(s / np.float32(f.size))


def contains_nan(field_global: np.ndarray) -> bool:
    return bool(np.isnan(np.asarray(field_global, dtype=np.float32)).any())


def fmt(v) -> str:
    """std::ostream << float with default flags: %g, 6 significant digits."""
    return "%g" % float(v)


def time_block(kind: str, time_step: int, names: Sequence[str], fields: np.ndarray) -> List[str]:
    """The lines fieldCalculate prints for one saved time."""
    out = [f"Time: {time_step}", "{"]
    if kind == "containsNaN":
        bad = [n for n, f in zip(names, fields) if contains_nan(f)]
        out += [f"    NaN detected in field {n}" for n in bad]
        out.append("    No NaN values detected in any field." if not bad else
                   f"    Total number of fields with NaN values: {len(bad)}")
    else:
        out += [f"    mean({n}): {fmt(spatial_mean(f))};" for n, f in zip(names, fields)]
    return out + ["};", ""]
