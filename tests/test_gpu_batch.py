"""Config 3 at full size: 16 seeded config-2 variants of uneven size (10k-2M
triangles, 256^2 to 1920x1080, 4-64 spp, depth 8-12) rendered in one
mrtxRenderBatch submission. Every job's FP64 accumulation must equal, bit for
bit, the same job rendered alone with mrtxRenderFrames: batching runs the
jobs' waves together in one set of kernel launches but changes none of their
samples."""
import numpy as np
import pytest

from miniraytrace_b200 import scenes

pytestmark = pytest.mark.gpu


def test_batch_of_uneven_jobs_equals_each_job_alone(gpu):
    jobs = scenes.batch_jobs()
    engines = []
    for s in jobs:
        e = gpu.Engine(s.settings["width"], s.settings["height"])
        s.apply(e)
        engines.append(e)
    infos = gpu.render_batch(engines, [s.spp for s in jobs])
    assert [i["spp"] for i in infos] == [s.spp for s in jobs]
    # one set of launches for all jobs: every engine reports the batch's
    # launches and device time, fewer launches than the jobs alone
    stats = [e.stats() for e in engines]
    assert len({st["kernelLaunches"] for st in stats}) == 1
    assert len({st["lastRenderMs"] for st in stats}) == 1
    assert all(st["batchJobs"] == len(jobs) for st in stats)
    batch_launches = stats[0]["kernelLaunches"]
    batched = []
    for e in engines:
        acc, n = e.read_accumulation()
        batched.append((acc, n))
        e.close()
    alone_launches = 0
    for s, (acc, n) in zip(jobs, batched):
        e = gpu.Engine(s.settings["width"], s.settings["height"])
        s.apply(e)
        e.render_frames(s.spp)
        ref, m = e.read_accumulation()
        st = e.stats()
        assert st["batchJobs"] == 1
        alone_launches += st["kernelLaunches"]
        e.close()
        assert n == m == s.spp, s.name
        assert np.array_equal(acc, ref), s.name
    assert batch_launches * 4 < alone_launches


def test_batch_argument_checks_and_repeats(gpu):
    s = scenes.box_sphere(32, 32)
    a, b = gpu.Engine(32, 32), gpu.Engine(32, 32)
    s.apply(a)
    s.apply(b)
    # queued single frames render before the batch's samples, in order
    a.render_frame()
    infos = gpu.render_batch([a, b], [3, 4])
    assert [i["spp"] for i in infos] == [4, 4]
    assert np.array_equal(a.read_accumulation()[0], b.read_accumulation()[0])
    # the same engine twice gets both shares
    infos = gpu.render_batch([a, a], [1, 2])
    assert a.read_accumulation()[1] == 7
    assert gpu.render_batch([], []) == []
    a.close()
    b.close()
