"""Learned-closure study: an under-resolved D3Q27 lid-driven cavity on a
coarse grid, with and without the learned relaxation-time correction, measured
against a fine run at twice the resolution.

    python -m cudalbm_b200.closure_study [--nc 128] [--coarse-steps 10000] [--seeds 8]
        [--snapshots 6] [--stride 3] [--json out.json]

Steps (all on the GPU through the library):
 1. Training data: ``seeds`` fine runs (2 nc per edge) of the lid-driven
    cavity with initial velocities perturbed by U(-1e-3, 1e-3); at
    ``snapshots`` times each is box-filtered 2:1 onto the coarse grid (the
    non-equilibrium stress rescaled to the coarse lattice), the coarse solver
    takes one step from it, and every ``stride``-th interior node gives a
    sample (16 features, target dtau; lbm_trainer_add).  With ``window`` > 1
    each sample's dtau is fitted to that many consecutive coarse steps, each
    from the filtered fine state (lbm_trainer_add_window).
 2. Training: 16 -> 32 -> 32 -> 1 GELU network, Adam, on the GPU.
 3. Calibration: the network's output is shrunk by the factor in
    ``shrink`` that minimises the centreline error of a coarse run against
    one more perturbed fine run (seed ``seeds``, not used for training) --
    never against the evaluation case.
 4. Evaluation: the unperturbed case.  Plain coarse, learned coarse and the
    fine run (the truth) advance the same physical time (coarse steps =
    fine steps / 2 at equal lattice velocity).  Errors: centreline u(y) at
    x = z = mid and the whole velocity field, relative L2, against the fine
    run box-filtered 2:1 (the stated measure) and against the fine run sampled
    at the coarse nodes' positions (trilinear; the 2:1 box filter places the
    coarse wall rows a quarter fine cell inside the walls).  Wall times of
    the coarse runs and of the fine run over the same physical time.

The coarse relaxation time defaults to 0.5077, the value of the 512^3,
Re = 10000 configuration this reproduces at reduced size (Re follows from
it: Re = u_lid (nc - 1) / ((tau - 0.5) / 3)).
"""
from __future__ import annotations

import argparse
import json
import time
from typing import Callable, Dict, Sequence

import numpy as np

from . import _lib
from .closure import Trainer, mlp_infer, save_mlp
from .solver import Cavity


def centreline(m: np.ndarray) -> np.ndarray:
    """u(y) at x = z = mid of moments [10][nz][ny][nx] (mean of the four
    middle columns for an even edge), in lattice units."""
    n = m.shape[1]
    lo, hi = (n - 1) // 2, n // 2
    return 0.25 * (m[1, lo, :, lo] + m[1, lo, :, hi] + m[1, hi, :, lo] + m[1, hi, :, hi]) / 3.0


def centreline_at_coarse_nodes(fine: Cavity, nc: int) -> np.ndarray:
    """``centreline`` of the fine run sampled at the coarse nodes' positions
    (trilinear): two device cut planes at the coarse middle z positions,
    interpolated in x and y here -- no full read of the fine field."""
    nf = fine.shape[0]
    lo, hi = (nc - 1) // 2, nc // 2
    y = np.arange(nc) * (nf - 1) / (nc - 1)
    j0 = np.minimum(np.floor(y).astype(int), nf - 2)
    wy = y - j0
    cols = []
    for k in (lo, hi):
        u = fine.cut_plane(2, k / (nc - 1))[1].astype(np.float64)  # [ny][nx] at z of coarse plane k
        for i in (lo, hi):
            x = i * (nf - 1) / (nc - 1)
            i0 = min(int(np.floor(x)), nf - 2)
            wx = x - i0
            ux = u[:, i0] * (1 - wx) + u[:, i0 + 1] * wx
            cols.append(ux[j0] * (1 - wy) + ux[j0 + 1] * wy)
    return 0.25 * sum(cols) / 3.0


def sample_at_coarse_nodes(fine_vel: np.ndarray, nc: int) -> np.ndarray:
    """Fine velocity [3][nf][nf][nf] at the coarse node positions (trilinear)."""
    nf = fine_vel.shape[1]
    x = np.arange(nc) * (nf - 1) / (nc - 1)
    i0 = np.minimum(np.floor(x).astype(int), nf - 2)
    w = x - i0
    out = []
    for a in fine_vel.astype(np.float64):
        a = a[:, :, i0] * (1 - w) + a[:, :, i0 + 1] * w
        a = a[:, i0, :] * (1 - w)[None, :, None] + a[:, i0 + 1, :] * w[None, :, None]
        a = a[i0] * (1 - w)[:, None, None] + a[i0 + 1] * w[:, None, None]
        out.append(a)
    return np.stack(out)


def rel(a, b) -> float:
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def run_study(nc: int = 128, lattice: int = 27, u_lid: float = 0.05, tau_coarse: float = 0.5077,
              coarse_steps: int = 10000, seeds: int = 8, snapshots: int = 6, stride: int = 3,
              min_neq: float = 3e-4, train_steps: int = 3000, batch: int = 16384, lr: float = 2e-3,
              dtau_range: Sequence[float] = (0.0, 0.05), shrink: Sequence[float] = (1.0, 0.5, 0.25),
              device: int = 0, save: str = "", field_pos_max: int = 512, window: int = 1,
              log: Callable[[str], None] = print) -> Dict[str, object]:
    """``field_pos_max``: largest fine edge for which the whole fine field is
    read back to sample it at the coarse nodes (field_pos); above it only
    the centreline is sampled (two device cut planes)."""
    nf = 2 * nc
    Re = u_lid * (nc - 1) / ((tau_coarse - 0.5) / 3.0)
    Tc, Tf = int(coarse_steps), 2 * int(coarse_steps)
    snaps = [int(Tf * (k + 1) / (snapshots + 1)) for k in range(snapshots)]
    cav = lambda n: Cavity(lattice, n, n, n, Re, u_lid, device=device)
    whole_field = nf <= field_pos_max

    def fine_run(seed, trainer=None, truth_at=()):
        """Fine run to Tf; samples at the snapshots, filtered states at truth_at."""
        out = {}
        with cav(nf) as f, cav(nc) as c:
            f.init_regions()
            if nf >= 512:
                f.autotune(3)
            if seed is not None:
                f.perturb_velocity(1e-3, seed)
            f.synchronize()
            t0 = time.perf_counter()
            done = 0
            for s in sorted(set(snaps if trainer is not None else []) | set(truth_at)):
                f.step(s - done)
                done = s
                if s in truth_at:
                    c.filter_from(f)
                    out[s // 2] = (c.read(), centreline_at_coarse_nodes(f, nc),
                                   sample_at_coarse_nodes(f.read()[1:4], nc) if whole_field else None)
                if trainer is not None and s in snaps:
                    c.filter_from(f)
                    if window == 1:
                        f.step(2)
                        trainer.add(c, f, stride=stride, min_neq=min_neq)
                    else:  # one dtau per node fitted to `window` coarse steps
                        trainer.add_window(c, f, window, stride=stride, min_neq=min_neq)
                    done += 2 * window
            f.step(Tf - done)
            f.synchronize()
            out["wall"] = time.perf_counter() - t0
        return out

    def coarse_run(net, truth, times=(Tc // 2, Tc), dtau=False):
        res = {}
        with cav(nc) as c:
            c.init_regions()
            if net is not None:
                c.set_closure(net)
            c.step(2)
            c.synchronize()
            t0 = time.perf_counter()
            done = 2
            walls = 0.0
            for t in times:
                c.step(t - done)
                c.synchronize()
                walls = time.perf_counter() - t0
                done = t
                m = c.read()
                jb, jc, ji = truth[t]
                res[t] = {"centreline_box": rel(centreline(m), centreline(jb)),
                          "field_box": rel(m[1:4], jb[1:4]),
                          "centreline_pos": rel(centreline(m), jc),
                          "field_pos": rel(m[1:4], ji) if ji is not None else None}
            res["wall"] = walls
            res["steps"] = Tc - 2
            if dtau:
                dt = c.closure_dtau()
                res["dtau"] = {"mean": float(dt.mean()), "max": float(dt.max()),
                               "nonzero_fraction": float((dt != 0).mean())}
        return res

    t0 = time.perf_counter()
    trainer = Trainer(capacity=max(1_000_000, int(1.2 * seeds * snapshots * (nc - 2) ** 3 / stride)), device=device)
    for seed in range(seeds):
        fine_run(seed, trainer)
    gen_s = time.perf_counter() - t0
    feats, targ = trainer.samples()
    log(f"samples {len(targ)} in {gen_s:.1f} s; target percentiles 5/50/95 {np.percentile(targ, [5, 50, 95])}")
    t0 = time.perf_counter()
    net, rep = trainer.fit(steps=train_steps, batch=batch, lr=lr, dtau_lo=dtau_range[0], dtau_hi=dtau_range[1])
    train_s = time.perf_counter() - t0
    k = max(1, len(targ) // 10)
    pred = mlp_infer(net, feats[-k:], tensor_cores=True, device=device) * net.out_scale
    tk = np.clip(targ[-k:], dtau_range[0], dtau_range[1])
    r2 = float(1.0 - np.mean((pred - tk) ** 2) / np.var(tk))
    log(f"trained {train_steps} steps in {train_s:.1f} s: loss {rep['loss_first']:.3f} -> {rep['loss_last']:.3f}, "
        f"R2 on the last tenth of the samples {r2:.3f}")
    trainer.close()

    # calibration on a held-out perturbed seed
    calib = fine_run(seeds, truth_at=(Tf,))
    base = net.out_scale
    scores = {}
    for a in shrink:
        net.out_scale = base * a
        scores[a] = coarse_run(net, calib, times=(Tc,))[Tc]["centreline_box"]
    best = min(scores, key=scores.get)
    net.out_scale = base * best
    log(f"calibration (centreline error on seed {seeds}): {scores} -> shrink {best}")

    truth = fine_run(None, truth_at=(Tf // 2, Tf))
    plain = coarse_run(None, truth)
    learned = coarse_run(net, truth, dtau=True)
    if save:
        save_mlp(save, net)
    out = {
        "config": {"lattice": f"D3Q{lattice}", "coarse": nc, "fine": nf, "Re": Re, "tau_coarse": tau_coarse,
                   "u_lid": u_lid, "coarse_steps": Tc, "fine_steps": Tf, "seeds": seeds, "snapshots": snapshots,
                   "stride": stride, "min_neq": min_neq, "dtau_range": list(dtau_range), "window": window},
        "training": {"samples": int(len(targ)), "generation_s": gen_s, "train_s": train_s, "steps": train_steps,
                     "loss_first": rep["loss_first"], "loss_last": rep["loss_last"], "r2_held_out": r2,
                     "shrink_scores": {str(k): v for k, v in scores.items()}, "shrink": best},
        "plain": plain, "learned": learned,
        "fine_wall_s": truth["wall"],
        "speedup_learned_vs_fine": truth["wall"] / learned["wall"],
        "dtau": learned.pop("dtau"),
    }
    for t in (Tc // 2, Tc):
        log(f"t={t}: plain {plain[t]}  learned {learned[t]}")
    log(f"wall: fine {truth['wall']:.2f} s, coarse plain {plain['wall']:.2f} s, coarse learned {learned['wall']:.2f} s")
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--nc", type=int, default=128)
    ap.add_argument("--coarse-steps", type=int, default=10000)
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--snapshots", type=int, default=6)
    ap.add_argument("--stride", type=int, default=3, help="every stride-th interior node is a sample")
    ap.add_argument("--dtau-range", default="0,0.05", help="clip of the targets and of the output, lo,hi")
    ap.add_argument("--shrink", default="1,0.5,0.25", help="output scale factors tried in the calibration "
                    "(0 = the plain method)")
    ap.add_argument("--window", type=int, default=1, help="coarse steps each sample's dtau is fitted to (1: one step)")
    ap.add_argument("--save", default="", help="write the trained network (.npz)")
    ap.add_argument("--json", default="", help="write the results")
    a = ap.parse_args()
    res = run_study(nc=a.nc, coarse_steps=a.coarse_steps, seeds=a.seeds, train_steps=a.train_steps,
                    snapshots=a.snapshots, stride=a.stride, save=a.save,
                    dtau_range=[float(v) for v in a.dtau_range.split(",")],
                    shrink=[float(v) for v in a.shrink.split(",")], window=a.window)
    text = json.dumps(res, indent=1, default=float)
    if a.json:
        with open(a.json, "w") as fh:
            fh.write(text)
    print(text)


if __name__ == "__main__":
    main()
