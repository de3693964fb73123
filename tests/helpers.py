"""Shared helpers for the test-suite: golden fixtures and error metrics."""
from __future__ import annotations

import json
import os

import numpy as np

from cudalbm_b200 import casefiles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["q19_16c_re100", "q27_16c_re100", "q19_24x16x8_fo", "q27_16x24x32_fo", "q19_16c_lidic"]


def load_golden(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    meta = json.loads(str(g["meta"]))
    arrays = {k: g[k] for k in g.files if k != "meta"}
    return meta, arrays


def spec_of(meta):
    return casefiles.CaseSpec(**meta["spec"])


def lattice_q(meta):
    return 19 if meta["lattice"] == "D3Q19" else 27


def rel_l2(a, b):
    """Per-field relative L2 error ||a-b|| / ||b|| over the trailing axes."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    axes = tuple(range(1, a.ndim))
    num = np.sqrt(np.sum((a - b) ** 2, axis=axes))
    den = np.sqrt(np.sum(b ** 2, axis=axes))
    return num / np.maximum(den, 1e-300)


def max_abs(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.max(np.abs(a - b), axis=tuple(range(1, a.ndim)))


def read_vts(path):
    """Minimal reader of the VTK XML structured-grid files fieldConvert writes
    (appended raw data, UInt64 block headers): (extent, {name: values}, points)."""
    import re

    raw = open(path, "rb").read()
    mark = raw.index(b'<AppendedData encoding="raw">_') + len(b'<AppendedData encoding="raw">_')
    head = raw[:mark].decode()
    extent = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', head).group(1).split()]
    arrays = re.findall(r'<DataArray type="Float32" Name="([^"]+)"(?: NumberOfComponents="3")? format="appended" '
                        r'offset="(\d+)"/>', head)
    out, points = {}, None
    for name, off in arrays:
        p = mark + int(off)
        nbytes = int(np.frombuffer(raw[p:p + 8], dtype="<u8")[0])
        vals = np.frombuffer(raw[p + 8:p + 8 + nbytes], dtype="<f4")
        if name == "Coordinates":
            points = vals.reshape(-1, 3)
        else:
            out[name] = vals
    assert raw.endswith(b"</AppendedData>\n</VTKFile>\n")
    return extent, out, points
