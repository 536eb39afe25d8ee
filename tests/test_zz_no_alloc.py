"""mrtxBuildEnvCdfNoAlloc: the environment CDF from device memory into device
memory with its scratch in a static device array (no allocation inside the
call). Its results must equal mrtxBuildEnvCdf's (the engine path, itself
bit-exact with the reference's sequential sums) on every call, including
back-to-back calls that reuse the same scratch.

Tolerance: none. Both entry points run the same kernels on the same inputs
in the same order, so the CDF and the integral must match bit for bit.

Torch only provides the test's device buffers and streams; the library call
goes through the C ABI (ctypes)."""
import numpy as np
import pytest

from miniraytrace_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def device_buffers(torch, sky):
    h, w = sky.shape[:2]
    tex = torch.from_numpy(np.ascontiguousarray(sky, np.float32)).cuda()
    cdf = torch.full((w * h + h,), float("nan"), dtype=torch.float32, device="cuda")
    integ = torch.full((1,), float("nan"), dtype=torch.float32, device="cuda")
    return tex, cdf, integ


@pytest.mark.parametrize("w,h", [(2048, 1024), (64, abi.ENV_CDF_NOALLOC_MAX_HEIGHT)])
def test_matches_engine_path_on_consecutive_calls(gpu, w, h):
    import torch
    sky = scenes.procedural_sky(w, h)
    e = gpu.Engine(16, 16)
    ref_cdf, ref_integ = e.build_env_cdf(sky)
    e.close()
    tex, cdf, integ = device_buffers(torch, sky)
    stream = torch.cuda.Stream()
    for call in range(2):
        cdf.fill_(float("nan"))
        integ.fill_(float("nan"))
        torch.cuda.synchronize()
        gpu.build_env_cdf_no_alloc(tex.data_ptr(), w, h, cdf.data_ptr(), integ.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        got = cdf.cpu().numpy()
        assert np.array_equal(got, ref_cdf), (call, int(np.sum(got != ref_cdf)))
        assert np.float32(integ.item()) == np.float32(ref_integ), call


def test_scratch_reuse_across_sizes_and_default_stream(gpu):
    """A smaller map after a larger one: stale scratch rows must not leak."""
    import torch
    e = gpu.Engine(16, 16)
    # heights at, just past and below the 1,000-row parameter chunks
    for w, h in ((512, 4096), (300, 100), (300, 100), (64, 1000), (64, 1001), (96, 2000)):
        sky = scenes.procedural_sky(w, h, sun_azim_deg=float(w % 90))
        ref_cdf, ref_integ = e.build_env_cdf(sky)
        tex, cdf, integ = device_buffers(torch, sky)
        torch.cuda.synchronize()
        gpu.build_env_cdf_no_alloc(tex.data_ptr(), w, h, cdf.data_ptr(), integ.data_ptr(), 0)
        torch.cuda.synchronize()
        assert np.array_equal(cdf.cpu().numpy(), ref_cdf), (w, h)
        assert np.float32(integ.item()) == np.float32(ref_integ), (w, h)
    e.close()


def test_rejects_oversized_and_host_inputs(gpu):
    import torch
    h = abi.ENV_CDF_NOALLOC_MAX_HEIGHT + 1
    tex = torch.zeros((h, 2, 4), dtype=torch.float32, device="cuda")
    cdf = torch.zeros((2 * h + h,), dtype=torch.float32, device="cuda")
    integ = torch.zeros((1,), dtype=torch.float32, device="cuda")
    with pytest.raises(gpu.MrtError) as err:
        gpu.build_env_cdf_no_alloc(tex.data_ptr(), 2, h, cdf.data_ptr(), integ.data_ptr())
    assert err.value.code == abi.MRT_ERROR_INVALID_ARGUMENT
    assert str(abi.ENV_CDF_NOALLOC_MAX_HEIGHT) in str(err.value)
    host = np.zeros((4, 4, 4), np.float32)
    with pytest.raises(gpu.MrtError) as err:
        gpu.build_env_cdf_no_alloc(host.ctypes.data, 4, 4, cdf.data_ptr(), integ.data_ptr())
    assert err.value.code == abi.MRT_ERROR_INVALID_ARGUMENT
    assert "device memory" in str(err.value)


def test_rejects_misaligned_pointers_before_launching(gpu):
    """A texel pointer carved from a pool at a 4-byte offset would fault on
    the device's 16-byte loads; the call refuses it on the host instead, and
    the context stays usable for a correct call afterwards."""
    import torch
    w, h = 64, 32
    sky = scenes.procedural_sky(w, h)
    tex, cdf, integ = device_buffers(torch, sky)
    big = torch.zeros((h * w * 4 + 4,), dtype=torch.float32, device="cuda")
    for args in ((big.data_ptr() + 4, cdf.data_ptr(), integ.data_ptr()),
                 (tex.data_ptr(), cdf.data_ptr() + 2, integ.data_ptr()),
                 (tex.data_ptr(), cdf.data_ptr(), integ.data_ptr() + 1)):
        with pytest.raises(gpu.MrtError) as err:
            gpu.build_env_cdf_no_alloc(args[0], w, h, args[1], args[2])
        assert err.value.code == abi.MRT_ERROR_INVALID_ARGUMENT
        assert "aligned" in str(err.value)
    e = gpu.Engine(16, 16)
    ref_cdf, _ = e.build_env_cdf(sky)
    e.close()
    gpu.build_env_cdf_no_alloc(tex.data_ptr(), w, h, cdf.data_ptr(), integ.data_ptr(), 0)
    torch.cuda.synchronize()
    assert np.array_equal(cdf.cpu().numpy(), ref_cdf)
