"""Error table of the 16-bit moment storage (needs a GPU).

    python tests/precision_report.py [N] [steps] [oracle_steps]

D3Q19 lid-driven cavity, Re = 1000, u_lid = 0.05.  Prints, per moment, the
max and relative-L2 error of FP16 and BF16 storage against the FP32 path after
`steps` steps, and of all three against the FP64 CPU oracle after
`oracle_steps` steps (the oracle is slow: keep N^3 * oracle_steps modest).
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

from cudalbm_b200 import casefiles  # noqa: E402
from cudalbm_b200.solver import Cavity  # noqa: E402
from helpers import max_abs, rel_l2  # noqa: E402

NAMES = casefiles.MOMENT_NAMES


def run(n, steps, storage):
    with Cavity(19, n, n, n, 1000.0, 0.05, storage=storage) as c:
        c.init_regions()
        c.step(steps)
        c.synchronize()
        return c.read("moments")


def table(title, runs, ref):
    print(f"\n{title}\n")
    print("| moment | " + " | ".join(f"{k} max abs | {k} rel L2" for k in runs) + " |")
    print("|---|" + "---|---|" * len(runs))
    errs = {k: (max_abs(v, ref), rel_l2(v, ref)) for k, v in runs.items()}
    for i, nm in enumerate(NAMES):
        print(f"| {nm} | " + " | ".join(f"{errs[k][0][i]:.2e} | {errs[k][1][i]:.2e}" for k in runs) + " |")


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 128
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 10000
    ostep = int(sys.argv[3]) if len(sys.argv) > 3 else 1000
    ref32 = run(n, steps, "f32")
    table(f"D3Q19 {n}^3, Re 1000, {steps} steps: 16-bit storage against the FP32 path",
          {"fp16": run(n, steps, "f16"), "bf16": run(n, steps, "bf16")}, ref32)
    from pyoracle import Oracle

    o = Oracle(19, n, n, n, 1000.0, 0.05)
    m = o.initial(casefiles.scaled_region_values(casefiles.lid_cavity_values(0.05)))
    o.run(m, ostep)
    table(f"D3Q19 {n}^3, Re 1000, {ostep} steps: against the FP64 oracle",
          {"fp32": run(n, ostep, "f32"), "fp16": run(n, ostep, "f16"), "bf16": run(n, ostep, "bf16")}, m)


if __name__ == "__main__":
    main()
