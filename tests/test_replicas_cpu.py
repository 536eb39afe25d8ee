"""Multi-rank path on CPU: two gloo ranks, each rendering its stripe of the
samples (miniraytrace_b200.replicas) with the CPU oracle standing in for a
GPU, combined with the same reduce bench.py uses. The combined accumulation
must equal one rank rendering all samples, and a rank that dies must make the
other's next collective fail instead of waiting forever."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from miniraytrace_b200 import replicas

W, H, SPP_PER_RANK = 12, 10, 3


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def scene():
    import oracle
    from miniraytrace_b200 import scenes

    o = oracle.OracleScene(W, H)
    scenes.box_sphere(W, H).apply(o)
    o.commit()
    return o


def render_frames(o, frames):
    """FP64 accumulation (r, g, b sums, sample count) of the given frame
    indices, in the engine's buffer layout."""
    acc = np.zeros((H * W, 4), np.float64)
    for f in frames:  # per pixel, samples added in order, as the kernels do
        acc[:, :3] += o.render_f32_sum64(f, 1, threads=2)
        acc[:, 3] += 1.0
    return acc.reshape(H, W, 4)


def rank_main(rank, world, port, die, q):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
        if die and rank == 1:
            os._exit(3)  # leaves between steps, with no collective in flight
        o = scene()
        acc = render_frames(o, replicas.frames_of(rank, world, 0, SPP_PER_RANK))
        buf = torch.from_numpy(acc.copy())
        replicas.combine_accumulation(buf, dist)
        slowest = replicas.max_over_ranks(float(rank + 1), dist, "cpu")
        q.put((rank, "ok", buf.numpy() if rank == 0 else None, slowest))
        dist.destroy_process_group()
    except Exception as e:  # reported to the test, which decides
        q.put((rank, "error", repr(e), None))


def run_ranks(world, die=False, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, die, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for p in procs:
        p.join(timeout)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    while not q.empty():
        r, status, payload, slowest = q.get()
        results[r] = (status, payload, slowest)
    return results, [p.exitcode for p in procs]


def test_stripes_partition_the_sample_set():
    frames = sorted(f for r in range(4) for f in replicas.frames_of(r, 4, 0, 5))
    assert frames == list(range(20))
    assert replicas.frames_of(1, 2, 3, 2) == [7, 9]
    assert replicas.sample_stream(0, 1) == (0, 1)
    with pytest.raises(ValueError):
        replicas.sample_stream(2, 2)


def test_two_ranks_combine_to_the_single_rank_image(oracle_lib):
    results, codes = run_ranks(2)
    assert codes == [0, 0], (codes, results)
    assert results[0][0] == "ok" and results[1][0] == "ok", results
    combined = results[0][1]
    assert results[0][2] == results[1][2] == 2.0  # slowest rank's value on both
    single = render_frames(scene(), range(2 * SPP_PER_RANK))
    assert np.array_equal(combined[..., 3], single[..., 3])
    # the same FP32 paths summed in another order: equal to FP64 rounding
    np.testing.assert_allclose(combined[..., :3], single[..., :3], rtol=1e-12, atol=1e-12)


def test_a_dead_rank_fails_the_others_collective(oracle_lib):
    results, codes = run_ranks(2, die=True, timeout=90)
    assert codes[1] == 3
    # rank 0 learns of it from the collective (an error, not a hang)
    assert codes[0] == 0 and results.get(0, ("missing",))[0] == "error", (codes, results)
