"""Autotuner for the kernels' compile-time constants.

Usage (on a machine with the target GPU):

    python -m miniraytrace_b200.autotune [--rounds 2] [--steps 3] [--write]

The tunable constants are preprocessor defines of the CUDA sources:

- ``MRT_TRAV_MIN_BLOCKS``: resident blocks per SM the traversal kernels are
  compiled for (bounds their registers: 7 -> 72, 6 -> 80, 8 -> 64);
- ``MRT_TRI_PHASE_PCT``: percent of a warp's active lanes with pending leaf
  triangles that starts a warp-wide triangle phase;
- ``MRT_REFILL_IDLE``: idle lanes of a persistent traversal warp before it
  takes new rays from the queue;
- ``MRT_SHADE_THREADS``: threads per block of the shade kernel;
- ``MRT_SHADE_MIN_BLOCKS``: resident blocks per SM the shade kernel is
  compiled for (a register bound; 0: none, about 100 registers);
- ``MRT_SHADOW_OVERLAP``: 1 runs a bounce's shadow kernel on a second stream
  beside the next bounce's extend kernel, 0 runs every kernel in order;
- ``MRT_SHARED_STACK``: traversal stack entries per thread held in shared
  memory (the rest in local memory; 0: all in local memory).

The search is coordinate descent from the current values
(``miniraytrace_b200/tuned.json``, else the sources' defaults): for each
constant in turn every candidate value is built into its own directory
(``build(defines=..., lib=...)``) and timed by ``bench.py`` in a child
process that loads that build (``MRT_LIBRARY``); the best value is kept
before the next constant is tried, and the sweep repeats for ``--rounds``.
The objective is Mpaths/s of the 1080p terrain workload (scene resident)
over the median device time of the child's timed steps (``bench.py``'s
``step_device_ms``: the engine's CUDA-event time of its kernels, free of the
host jitter around the call); the starting point is measured once before
the search and discarded, since a fresh GPU's first run reads low. With
``--write`` the winner goes to ``tuned.json``, which ``build()`` applies;
every measurement is stored beside it.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

from . import build as mrt_build

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent

DEFAULTS = {"MRT_TRAV_MIN_BLOCKS": 7, "MRT_TRI_PHASE_PCT": 25, "MRT_REFILL_IDLE": 8, "MRT_SHADE_THREADS": 256,
            "MRT_SHADOW_OVERLAP": 1, "MRT_SHARED_STACK": 0, "MRT_SHADE_MIN_BLOCKS": 0}
SPACE = {
    "MRT_TRAV_MIN_BLOCKS": [6, 7, 8],
    "MRT_TRI_PHASE_PCT": [6, 9, 12, 18, 25, 50, 75],
    "MRT_REFILL_IDLE": [4, 6, 8, 10, 12, 16],
    "MRT_SHADE_THREADS": [128, 256, 512],
    "MRT_SHADOW_OVERLAP": [0, 1],
    "MRT_SHARED_STACK": [0, 8, 16],
    "MRT_SHADE_MIN_BLOCKS": [0, 2, 3],
}


def measure(defines: dict, workdir: Path, steps: int, warmup: int) -> float:
    """Mpaths/s of bench.py's default workload with a build of `defines`."""
    tag = "_".join(f"{k[4:].lower()}{v}" for k, v in sorted(defines.items()))
    bdir = workdir / tag
    lib = bdir / "libmrt.so"
    mrt_build.build(defines=defines, lib=lib, build_dir=bdir)
    env = dict(os.environ, MRT_LIBRARY=str(lib))
    cmd = [sys.executable, str(ROOT / "bench.py"), "--steps", str(steps), "--warmup", str(warmup),
           "--no-cpu-baseline", "--e2e-steps", "0", "--interactive-frames", "0", "--no-room"]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, cwd=str(ROOT), timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"bench failed for {defines}:\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    out = json.loads(line)
    # paths per second of device time: the engine's own CUDA-event time of
    # its kernels per step (the step time around the call adds host jitter)
    paths = out["config"]["width"] * out["config"]["height"] * out["config"]["spp_per_step"]
    return paths / (float(np.median(out["step_device_ms"])) / 1e3) / 1e6


def tune(rounds: int, steps: int, warmup: int, log=print) -> dict:
    current = dict(DEFAULTS)
    current.update(mrt_build.tuned_defines())
    results = []
    with tempfile.TemporaryDirectory(prefix="mrt_tune_") as tmp:
        work = Path(tmp)
        cache: dict[tuple, float] = {}

        def score(d):
            key = tuple(sorted(d.items()))
            if key not in cache:
                cache[key] = measure(d, work, steps, warmup)
                results.append({"defines": dict(d), "mpaths_per_s": cache[key]})
                log(json.dumps(results[-1]))
            return cache[key]

        measure(current, work, steps, warmup)  # a first run on a fresh GPU reads low: discarded
        best = score(current)
        for _ in range(rounds):
            changed = False
            for name, values in SPACE.items():
                for v in values:
                    if v == current[name]:
                        continue
                    cand = dict(current, **{name: v})
                    s = score(cand)
                    if s > best:
                        best, current, changed = s, cand, True
            if not changed:
                break
    return {"defines": current, "mpaths_per_s": best, "measurements": results,
            "objective": "Mpaths/s over the median device time per step, 1920x1080 terrain (2,420,738 triangles), 64 spp per step, "
                         f"{steps} timed steps after {warmup} warm-up steps"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--write", action="store_true", help="store the winner in tuned.json")
    a = ap.parse_args()
    res = tune(a.rounds, a.steps, a.warmup)
    print(json.dumps({"best": res["defines"], "mpaths_per_s": res["mpaths_per_s"]}))
    if a.write:
        mrt_build.TUNED.write_text(json.dumps(res, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
