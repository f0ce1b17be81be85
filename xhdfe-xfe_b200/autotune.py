"""Autotuner of the matvec form (b200fe_options.pass_kernel) per panel class.

The Schur system's matvec has four forms with the same answer to rounding
(b200fe.h: pass_kernel): 0 the explicit Schur block solved by the persistent
PCG where it applies (else the run-level pass), 1 the observation-level tile
pass, 2 the block-level pass with per-warp bins, 3 the run-level pass.  Which
is fastest depends on the panel: its size, its number of FE dims and how its
groups are spread (runs per segment, movers per firm).  This script times
every form on seeded AKM panels of each class (2 or 3 FE dims x size bucket)
with CUDA events around absorb_device and writes the fastest per class:

    python xhdfe-xfe_b200/autotune.py [--out xhdfe-xfe_b200/tuning.json]

make_options(pass_kernel="auto") then picks the form from the committed
table by the call's dims and rows (choose_pass_kernel): a table lookup, so
the choice, and the answer, do not depend on timing at run time.
"""

from __future__ import annotations

import argparse
import json
import math
import statistics
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
TABLE = HERE / "tuning.json"
FORMS = (0, 1, 2, 3)
# size buckets: bucket b holds panels of [10^b, 10^(b+1)) rows; the panel timed
# for a bucket has 3 * 10^b rows (2 * 10^7 for the largest)
BUCKETS = (4, 5, 6, 7)


def bucket_of(n: int) -> int:
    """Size bucket of a panel of n rows, clamped to the tuned range."""
    b = int(math.floor(math.log10(n))) if n > 0 else BUCKETS[0]
    return min(max(b, BUCKETS[0]), BUCKETS[-1])


def load_table(path: Path = TABLE) -> dict:
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def choose_pass_kernel(num_dims: int, n: int, table: dict | None = None) -> int:
    """The tuned form for a panel of num_dims FE dims and n rows; 0 (the
    library's default) where the table has no entry."""
    t = load_table() if table is None else table
    key = f"dims{min(max(num_dims, 2), 3)}_b{bucket_of(n)}"
    entry = t.get("classes", {}).get(key)
    return int(entry["pass_kernel"]) if entry else 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(TABLE))
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args(argv)
    sys.path.insert(0, str(HERE.parent))
    import numpy as np
    import torch

    import __graft_entry__ as ge
    pkg = ge.load_package()
    panels = ge.load_module("panels")
    dev = torch.device("cuda", 0)
    ab = pkg.Absorber(0)
    classes = {}
    for dims in (2, 3):
        for b in BUCKETS:
            n = int(3 * 10 ** b) if b < 7 else 20_000_000
            p = panels.akm_two_way(n, n_firms=max(100, n // 60), seed=17 + b, three_way=dims == 3)
            p = panels.subset(p, panels.drop_singletons(p.fes))
            v = torch.empty((p.k + 1, p.n), dtype=torch.float64, device=dev)
            v[0].copy_(torch.from_numpy(p.y))
            v[1:].copy_(torch.from_numpy(np.ascontiguousarray(p.X.T)))
            g = [torch.from_numpy(np.ascontiguousarray(f)).to(dev) for f in p.fes]
            times = {}
            for form in FORMS:
                o = pkg.make_options(tol=1e-8, pass_kernel=form)
                ab.absorb_device(v, g, p.levels, None, o)  # warm-up of this shape
                ms = []
                for _ in range(a.reps):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    torch.cuda.synchronize()
                    e0.record()
                    ab.absorb_device(v, g, p.levels, None, o)
                    e1.record()
                    torch.cuda.synchronize()
                    ms.append(e0.elapsed_time(e1))
                times[str(form)] = statistics.median(ms)
            best = min(FORMS, key=lambda f: times[str(f)])
            key = f"dims{dims}_b{b}"
            classes[key] = {"pass_kernel": best, "rows": p.n, "levels": list(map(int, p.levels)),
                            "ms": times}
            print(json.dumps({key: classes[key]}), flush=True)
            del v, g
    ab.close()
    out = {"device": torch.cuda.get_device_name(0), "made": time.strftime("%Y-%m-%d"),
           "command": "python xhdfe-xfe_b200/autotune.py", "reps": a.reps,
           "workload": "seeded AKM panels (panels.akm_two_way, about 60 rows per firm), 3 columns, "
                       "tol 1e-8, mixed precision; device time of absorb_device (CUDA events)",
           "classes": classes}
    Path(a.out).write_text(json.dumps(out, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
