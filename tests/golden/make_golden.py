"""Generate the golden fixtures from the reference solvers themselves.

Runs the reference executables built from its own sources by
``oracle/Makefile.ref`` (``oracle/_ref/momentBasedD3Q19`` and
``oracle/_ref/momentBasedD3Q27``) on small lid-driven-cavity case directories
and stores their ``.LBMBin`` outputs as compressed ``.npz`` fixtures (global
x-fastest order, float32, exactly as written by the reference).

Needs a CUDA GPU (the reference has no CPU path).  Usage:

    python tests/golden/make_golden.py OUTDIR

The fixtures committed next to this script were produced by this command on
an NVIDIA B200.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from cudalbm_b200 import casefiles, lbmbin  # noqa: E402

FO_ALL = ("S", "SMean", "k", "kMean", "momentsMean")

# name -> (lattice, CaseSpec kwargs)
CASES = {
    "q19_16c_re100": ("D3Q19", dict(nx=16, ny=16, nz=16, Re=100.0, u_inf=0.05, n_steps=201,
                                    save_interval=200, info_interval=100)),
    "q27_16c_re100": ("D3Q27", dict(nx=16, ny=16, nz=16, Re=100.0, u_inf=0.05, n_steps=201,
                                    save_interval=200, info_interval=100)),
    "q19_24x16x8_fo": ("D3Q19", dict(nx=24, ny=16, nz=8, Re=400.0, u_inf=0.05, n_steps=101,
                                     save_interval=100, info_interval=100, function_objects=FO_ALL)),
    "q27_16x24x32_fo": ("D3Q27", dict(nx=16, ny=24, nz=32, Re=400.0, u_inf=0.05, n_steps=101,
                                      save_interval=100, info_interval=100, function_objects=FO_ALL)),
    "q19_16c_lidic": ("D3Q19", dict(nx=16, ny=16, nz=16, Re=1000.0, u_inf=0.0256, lid_ic=0.0064,
                                    n_steps=51, save_interval=50, info_interval=50)),
}

FO_FILES = {"S": "S", "SMean": "SMean", "k": "k", "kMean": "kMean", "momentsMean": "momentsMean"}


def run_case(name: str, lattice: str, kw: dict, outdir: str) -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", f"momentBased{lattice}")
    if not os.path.exists(exe):
        raise SystemExit(f"{exe} missing: build it with make -f oracle/Makefile.ref")
    spec = casefiles.CaseSpec(**kw)
    with tempfile.TemporaryDirectory() as case:
        casefiles.write_case(case, spec)
        proc = subprocess.run([exe, "-GPU", "0"], cwd=case, capture_output=True, text=True, timeout=600)
        if proc.returncode != 0:
            raise SystemExit(f"{name}: reference exited {proc.returncode}\n{proc.stdout[-2000:]}\n{proc.stderr[-2000:]}")
        t_end = spec.n_steps - 1 - ((spec.n_steps - 1) % spec.save_interval)
        arrays = {}
        mom = lbmbin.read(os.path.join(case, f"{spec.case_name}_{t_end}.LBMBin"))
        arrays["moments"] = mom.data.astype(np.float32)
        for fo in spec.function_objects:
            f = lbmbin.read(os.path.join(case, f"{FO_FILES[fo]}_{t_end}.LBMBin"))
            arrays[fo] = f.data.astype(np.float32)
        meta = dict(lattice=lattice, t=t_end, spec={k: v for k, v in kw.items()},
                    source="reference cudaLBM executables (oracle/_ref) on an NVIDIA B200")
        meta["spec"]["function_objects"] = list(spec.function_objects)
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), meta=json.dumps(meta), **arrays)
        print(f"{name}: t={t_end} fields={list(arrays)}")


def main() -> None:
    outdir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(outdir, exist_ok=True)
    for name, (lattice, kw) in CASES.items():
        run_case(name, lattice, kw, outdir)


if __name__ == "__main__":
    main()
