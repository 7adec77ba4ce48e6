"""tc_render_no_alloc: the render entry point for callers that cannot let the library allocate.

Hosts whose device memory all belongs to their own pool or framework allocator, or that run under
a fixed device-memory budget, cannot have a cudaMalloc made behind their allocator's back at render
time. They pass the output buffer themselves; the library's scratch lives in a static device
array. The sums it produces must equal those of tc_render + tc_readback_sums for the same scene,
parameters and seeds, on two consecutive calls (the second call shows that the shared scratch,
which keeps the first call's counters, is cleared between calls).
"""

import ctypes

import numpy as np
import pytest

from toaster_b200 import configs
from toaster_b200.scene import scene_to_gpu

pytestmark = pytest.mark.gpu


def test_render_no_alloc_matches_render_on_two_calls(native_lib):
    import torch

    from toaster_b200.renderer import GpuRenderer

    scene = configs.mixed(width=48, height=27, samples=16)
    with GpuRenderer(0) as r:
        r.upload(scene_to_gpu(scene))
        torch.cuda.synchronize()
        # A stream of the caller's own (torch's default stream is the legacy NULL stream, which
        # would select the context's stream instead).
        stream = torch.cuda.Stream(device=0)
        with torch.cuda.stream(stream):
            sums = torch.zeros(3 * scene.width * scene.height, dtype=torch.float64, device="cuda:0")
        for frame in (5, 6):
            r.render(samples=16, frame_index=frame)
            expected, _, n = r.readback_sums()
            assert n == 16
            params = r._params.copy()
            params["samples"] = 16
            params["frame_index"] = frame
            params["accumulated_samples"] = 0
            with torch.cuda.stream(stream):
                sums.fill_(123.0)  # stale contents: a new image must start from zero
            code = native_lib.tc_render_no_alloc(r._ctx, params.ctypes.data, ctypes.c_void_p(sums.data_ptr()),
                                                 sums.numel(), ctypes.c_void_p(stream.cuda_stream))
            r._check(code)
            stream.synchronize()
            got = sums.cpu().numpy().reshape(scene.height, scene.width, 3)
            assert np.allclose(got, expected, rtol=1e-12, atol=1e-12), np.abs(got - expected).max()
            assert got.sum() > 0


def test_render_no_alloc_rejects_a_short_buffer(native_lib):
    import torch

    from toaster_b200.native import TcError
    from toaster_b200.renderer import GpuRenderer

    scene = configs.mixed(width=16, height=9, samples=1)
    with GpuRenderer(0) as r:
        r.upload(scene_to_gpu(scene))
        short = torch.zeros(3 * 16 * 9 - 1, dtype=torch.float64, device="cuda:0")
        params = r._params.copy()
        code = native_lib.tc_render_no_alloc(r._ctx, params.ctypes.data, ctypes.c_void_p(short.data_ptr()),
                                             short.numel(), None)
        with pytest.raises(TcError, match="3 per pixel"):
            r._check(code)
