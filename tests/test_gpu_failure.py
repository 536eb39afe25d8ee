"""Failure paths, in forms that fault, trap or hang no GPU.

The failure is made on the host or by a bound the kernels already check:
  - a traversal visit budget set far too low (mrtxSetTraversalBudget): every
    ray that needs more node visits gives up, the kernel sets its error word
    and returns; the call that traced it must fail with MRT_ERROR_UNKNOWN
    (not hang, not return a silently wrong image), reset the accumulation,
    and leave the engine usable;
  - allocation failures injected into the library's own allocation calls
    (mrtxInjectAllocationFailure): engine creation, commits and renders that
    meet one return MRT_ERROR_OUT_OF_MEMORY, and once the injection is off
    the same engine renders exactly what a fresh engine renders.
The reference has neither: its device errors abort the process
(core/src/gpu/GpuContext.hpp:22-31) and std::bad_alloc becomes
MRT_ERROR_OUT_OF_MEMORY at the C ABI (capi/src/capi.cpp:116-120).

Tolerance: none. After recovery the accumulation must equal a fresh
engine's bit for bit (same scene, same sample streams)."""
import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

pytestmark = pytest.mark.gpu
W, H, SPP = 64, 48, 4


def fresh_accumulation(gpu, s):
    e = gpu.Engine(W, H)
    s.apply(e)
    e.render_frames(SPP)
    acc, spp = e.read_accumulation()
    e.close()
    assert spp == SPP
    return acc


def test_visit_budget_exhausted_is_an_error_not_a_hang(gpu):
    s = scenes.box_sphere(W, H)
    want = fresh_accumulation(gpu, s)
    e = gpu.Engine(W, H)
    s.apply(e)
    e.commit()
    e.set_traversal_budget(1)  # the TLAS root, then nothing
    with pytest.raises(gpu.MrtError) as err:
        e.render_frames(SPP)
    assert err.value.code == abi.MRT_ERROR_UNKNOWN
    assert "budget" in str(err.value)
    assert e.read_accumulation()[1] == 0  # the failed samples were not kept
    # samples queued by mrtRenderFrame fail where they are rendered: the read
    for _ in range(2):
        e.render_frame()
    with pytest.raises(gpu.MrtError):
        e.read_framebuffer()
    # trace queries report it too
    o = np.tile(np.array([[0.0, 1.0, 3.6]], np.float32), (16, 1))
    d = np.tile(np.array([[0.0, -0.1, -1.0]], np.float32), (16, 1))
    with pytest.raises(gpu.MrtError):
        e.trace_rays(o, d)
    # back to the default budget: the same engine renders the fresh image
    e.set_traversal_budget(0)
    e.render_frames(SPP)
    acc, spp = e.read_accumulation()
    assert spp == SPP
    assert np.array_equal(acc, want)
    e.close()


def test_engine_creation_meets_allocation_failure(gpu):
    gpu.inject_allocation_failure(0)
    try:
        with pytest.raises(gpu.MrtError) as err:
            gpu.Engine(W, H)
        assert err.value.code == abi.MRT_ERROR_OUT_OF_MEMORY
    finally:
        gpu.inject_allocation_failure(-1)
    e = gpu.Engine(W, H)
    e.close()


def test_commit_and_render_recover_from_allocation_failures(gpu):
    """Failures at successive allocations of a first commit and of the
    first render's wave state; each time the engine must come back."""
    s = scenes.box_sphere(W, H)
    want = fresh_accumulation(gpu, s)
    failed_commits = failed_renders = 0
    for succeed in (0, 1, 2, 3, 5, 8, 13, 21, 34):
        e = gpu.Engine(W, H)
        s.apply(e)
        gpu.inject_allocation_failure(succeed)
        try:
            try:
                e.commit()
            except gpu.MrtError as err:
                assert err.code == abi.MRT_ERROR_OUT_OF_MEMORY, err
                failed_commits += 1
            try:
                e.render_frames(SPP)
            except gpu.MrtError as err:
                assert err.code == abi.MRT_ERROR_OUT_OF_MEMORY, err
                failed_renders += 1
        finally:
            gpu.inject_allocation_failure(-1)
        e.reset_accumulation()
        e.render_frames(SPP)
        acc, spp = e.read_accumulation()
        assert spp == SPP
        assert np.array_equal(acc, want), succeed
        e.close()
    assert failed_commits >= 3 and failed_renders >= 1, (failed_commits, failed_renders)
