"""Train the learned warm start on converged solutions of the plain solver.

Workload: seeded synthetic AKM panels (panels.warmstart_panel_spec): N
log-uniform in [n_min, n_max], 2-4 FE dims (worker, firm, year, firm x year),
move probability 0.02-0.3, firm-size Zipf exponent 0.8-1.5, the outcome plus
12 regressors.  The first panels are training panels: the plain FP64 solver
solves each tightly and the features and targets of (a random subset of) its
levels are collected on the device; the network is trained by the library's
own BF16 forward/backward kernels and Adam.  The remaining panels are held
out: each is absorbed to tol 1e-8 (mixed precision, the default) cold, warm
(start from the prediction) and warm with the learned Jacobi scaling, and the
iterations, device milliseconds and the difference between the warm and cold
within transforms are reported.

    python xhdfe-xfe_b200/train_warmstart.py [--panels 200 --held-out 40]
        [--n-min 100000 --n-max 20000000] [--out xhdfe-xfe_b200/warmstart_mlp.npz]
        [--report PATH.json]

Writes the trained parameters (npz: params, plus training metadata) and a
JSON report of the held-out comparison.
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402


def to_device(p, dev):
    import torch
    v = torch.empty((p.k + 1, p.n), dtype=torch.float64, device=dev)
    v[0].copy_(torch.from_numpy(p.y))
    v[1:].copy_(torch.from_numpy(np.ascontiguousarray(p.X.T)))
    gids = [torch.from_numpy(np.ascontiguousarray(f)).to(dev) for f in p.fes]
    return v, gids


def timed_absorb(ab, v, gids, levels, opts):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    out, r = ab.absorb_device(v, gids, levels, None, opts)
    e1.record()
    torch.cuda.synchronize()
    return out, r, e0.elapsed_time(e1)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--panels", type=int, default=200)
    ap.add_argument("--held-out", type=int, default=40)
    ap.add_argument("--n-min", type=int, default=100_000)
    ap.add_argument("--n-max", type=int, default=20_000_000)
    ap.add_argument("--per-panel", type=int, default=100_000, help="training samples kept per panel")
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "warmstart_mlp.npz"))
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    import torch

    pkg = ge.load_package()
    panels = ge.load_module("panels")
    learned = pkg.learned
    dev = torch.device("cuda", 0)
    ab = pkg.Absorber(0)
    n_train = a.panels - a.held_out
    feats, targs, t_gen, t_collect = [], [], 0.0, 0.0
    rng = np.random.default_rng(a.seed)
    for i in range(n_train):
        spec = panels.warmstart_panel_spec(i, seed=a.seed, n_min=a.n_min, n_max=a.n_max)
        t0 = time.perf_counter()
        p = panels.warmstart_panel(spec)
        t_gen += time.perf_counter() - t0
        v, gids = to_device(p, dev)
        t0 = time.perf_counter()
        f, t, r = learned.collect_samples(ab, v, gids, p.levels)
        t_collect += time.perf_counter() - t0
        if f.shape[0] > a.per_panel:
            idx = torch.from_numpy(rng.choice(f.shape[0], a.per_panel, replace=False)).to(dev)
            f, t = f.index_select(0, idx), t.index_select(0, idx)
        feats.append(f.clone())
        targs.append(t.clone())
        del v, gids
    X = torch.cat(feats)
    T = torch.cat(targs)
    t0 = time.perf_counter()
    params = learned.train(ab, X, T, epochs=a.epochs, lr=a.lr, seed=a.seed,
                           log=lambda m: print(m, flush=True))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    _, final_loss = learned.grad(ab, torch.from_numpy(params).to(dev), X[:200_000], T[:200_000])
    np.savez(a.out, params=params, train_panels=n_train, samples=int(X.shape[0]),
             final_loss=final_loss, seed=a.seed, n_min=a.n_min, n_max=a.n_max)
    print(f"trained on {X.shape[0]} samples of {n_train} panels in {t_train:.1f} s "
          f"(generation {t_gen:.1f} s, collection {t_collect:.1f} s); loss {final_loss:.5f}", flush=True)

    rows = []
    opts = pkg.make_options(tol=1e-8)
    for i in range(n_train, a.panels):
        spec = panels.warmstart_panel_spec(i, seed=a.seed, n_min=a.n_min, n_max=a.n_max)
        p = panels.warmstart_panel(spec)
        v, gids = to_device(p, dev)
        res = {}
        for name, mode in (("cold", 0), ("warm", 1), ("warm_scaled", 3)):
            learned.set_warm_start(ab, params if mode else None, mode)
            timed_absorb(ab, v, gids, p.levels, opts)  # warm-up of this shape
            out, r, ms = timed_absorb(ab, v, gids, p.levels, opts)
            res[name] = (out.clone(), r.iterations, ms, bool(r.converged), r.warm_columns)
        learned.set_warm_start(ab, None)
        scale = torch.linalg.vector_norm(v, dim=1)
        scale[scale == 0] = 1.0
        row = {"n": p.n, "dims": spec["dims"], "levels": p.levels, "move_prob": spec["move_prob"],
               "zipf": spec["zipf"]}
        for name in ("cold", "warm", "warm_scaled"):
            out, its, ms, conv, wc = res[name]
            row[name] = {"iterations": its, "ms": ms, "converged": conv, "warm_columns": wc}
            if name != "cold":
                d = torch.linalg.vector_norm(out - res["cold"][0], dim=1) / scale
                row[name]["max_rel_diff_vs_cold"] = float(d.max().item())
        rows.append(row)
        print(json.dumps(row), flush=True)
        del v, gids
    summary = {"train_panels": n_train, "held_out": len(rows), "samples": int(X.shape[0]),
               "final_loss": final_loss, "train_s": t_train}
    for name in ("cold", "warm", "warm_scaled"):
        summary[name] = {"iterations_mean": float(np.mean([r[name]["iterations"] for r in rows])),
                         "ms_total": float(np.sum([r[name]["ms"] for r in rows])),
                         "all_converged": all(r[name]["converged"] for r in rows)}
    print(json.dumps({"summary": summary}), flush=True)
    if a.report:
        Path(a.report).write_text(json.dumps({"summary": summary, "panels": rows}, indent=1))
    ab.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
