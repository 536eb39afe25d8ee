"""The autotuner's search without a GPU: coordinate descent over the
kernels' compile-time constants keeps a value only when it measures better,
tries every candidate of every constant, and never measures a configuration
twice. The measurement (a build of the variant plus a bench.py run on the
GPU) is replaced by a fake objective with a known optimum; and the build's
define handling is checked by building nothing but the command lines."""
import json

from miniraytrace_b200 import autotune, build


def test_coordinate_descent_finds_the_fake_optimum(monkeypatch):
    optimum = {"MRT_TRAV_MIN_BLOCKS": 6, "MRT_TRI_PHASE_PCT": 50, "MRT_REFILL_IDLE": 8, "MRT_SHADE_THREADS": 512,
               "MRT_SHADOW_OVERLAP": 0, "MRT_SHARED_STACK": 16, "MRT_SHADE_MIN_BLOCKS": 2}
    seen = []

    def fake_measure(defines, workdir, steps, warmup):
        key = tuple(sorted(defines.items()))
        assert key not in seen or len(seen) == 1, "measured twice"  # the discarded first run repeats the start
        seen.append(key)
        return 1000.0 - sum(abs(defines[k] - v) / max(v, 1) for k, v in optimum.items())

    monkeypatch.setattr(autotune, "measure", fake_measure)
    monkeypatch.setattr(build, "tuned_defines", lambda: {})
    res = autotune.tune(rounds=3, steps=1, warmup=1, log=lambda *_: None)
    assert res["defines"] == optimum
    assert res["mpaths_per_s"] == 1000.0
    assert all(set(m["defines"]) == set(autotune.DEFAULTS) for m in res["measurements"])
    json.dumps(res)  # what --write stores


def test_tuned_defines_reach_only_the_tuned_sources(tmp_path, monkeypatch):
    calls = []
    monkeypatch.setattr(build, "_run", lambda cmd: calls.append(cmd) or type("R", (), {"stderr": ""})())
    monkeypatch.setattr(build, "BUILD", tmp_path / "main")
    monkeypatch.setattr(build.shutil, "move", lambda a, b: None)
    monkeypatch.delenv("MRT_LIBRARY", raising=False)
    build.build(force=True, defines={"MRT_REFILL_IDLE": 16}, lib=tmp_path / "v" / "libmrt.so",
                build_dir=tmp_path / "v")
    nvcc = [c for c in calls if "-c" in c and c[c.index("-c") + 1].endswith(".cu")]
    assert nvcc
    for c in nvcc:
        src = c[c.index("-c") + 1]
        assert ("-DMRT_REFILL_IDLE=16" in c) == src.endswith("pathtrace.cu"), src
        obj = c[c.index("-o") + 1]
        assert obj.startswith(str(tmp_path / ("v" if src.endswith("pathtrace.cu") else "main"))), obj
