"""Scene files through the native loader on the GPU (needs a B200).

A scene file with a textured, smooth-shaded glTF mesh is loaded by tc_scene_load and uploaded
straight from the library's buffers (GpuRenderer.upload_file); its image must agree with the
oracle's render of the same file loaded by the Python loader, within the statistical band of the
image parity tests. The file renderer's PNG holds exactly the device-converted RGBA8 bytes.
"""

import numpy as np
import pytest

from parity_cases import textured_scene
from test_gpu_parity import statistical_parity
from toaster_b200.render_file import render_file
from toaster_b200.scene import _decode_png, load_scene
from toaster_b200.stream import encode_png

pytestmark = pytest.mark.gpu


def test_scene_file_image_matches_oracle(renderer, tmp_path):
    path = textured_scene(tmp_path)
    statistical_parity(renderer, "textured_scene_file", scene=load_scene(path),
                       upload=lambda: renderer.upload_file(path))


def test_render_file_writes_the_device_converted_bytes(renderer, tmp_path):
    path = textured_scene(tmp_path)
    exposure = renderer.upload_file(path)
    assert exposure == 0.5
    renderer.render(samples=16, frame_index=3)
    rgba = renderer.readback_rgba8(exposure)
    w, h, ch, img = _decode_png(encode_png(rgba))
    assert (w, h, ch) == (48, 32, 4) and np.array_equal(img, rgba)
    out = render_file(path, tmp_path / "frame.png", spp=16)
    w, h, ch, img = _decode_png((tmp_path / "frame.png").read_bytes())
    assert (w, h) == (48, 32) and img[..., 3].min() == 255 and img[..., :3].max() > 0
    assert out["samples"] == 16
    jpg = render_file(path, tmp_path / "frame.jpg", spp=16)
    data = (tmp_path / "frame.jpg").read_bytes()
    assert data[:2] == b"\xff\xd8" and jpg["bytes"] == len(data)
