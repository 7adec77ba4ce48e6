"""Device JPEG frames (tc_encode_jpeg) and MJPEG streams of animation frames (needs a B200).

The encoder is not the reference's (the image crate's), so the bytes differ; the frames must be
valid baseline JPEGs that decode to the display image within JPEG error.
"""

import io

import numpy as np
import pytest
from PIL import Image

from toaster_b200 import configs
from toaster_b200.native import TcError
from toaster_b200.renderer import Animation, GpuRenderer
from toaster_b200.scene import scene_to_gpu
from toaster_b200.stream import mjpeg_part, split_mjpeg

pytestmark = pytest.mark.gpu


def psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10 * np.log10(255.0 ** 2 / max(mse, 1e-12))


def test_jpeg_frame_decodes_to_the_display_image(renderer):
    renderer.upload(scene_to_gpu(configs.mixed(width=320, height=180)))
    renderer.render(samples=32, max_bounces=6, frame_index=2)
    rgba = renderer.readback_rgba8(0.5)
    jpeg = renderer.encode_jpeg(quality=92, exposure_stops=0.5)
    assert jpeg[:2] == b"\xff\xd8" and jpeg[-2:] == b"\xff\xd9"
    img = np.asarray(Image.open(io.BytesIO(jpeg)).convert("RGB"))
    assert img.shape == (180, 320, 3)
    assert psnr(img, rgba[..., :3]) > 30.0
    low = renderer.encode_jpeg(quality=20, exposure_stops=0.5)
    assert len(low) < len(jpeg)


def test_jpeg_rejects_bad_quality(renderer):
    renderer.upload(scene_to_gpu(configs.plain_small()))
    renderer.render(samples=1)
    for q in (0, 101):
        with pytest.raises(TcError, match="JPEG quality must be between 1 and 100"):
            renderer.encode_jpeg(quality=q)


def test_mjpeg_stream_of_animation_frames(native_lib):
    anim = configs.BallisticAnimation(width=192, height=108, samples=4, max_bounces=4, frames=12)
    first = scene_to_gpu(anim.scene(0))
    stream = b""
    with GpuRenderer(0) as r:
        r.upload(first)
        with Animation(r, first, rebuild=True) as a:
            for k in range(0, 12, 4):
                rgba = a.frame(scene_to_gpu(anim.scene(k)), k)
                jpeg = r.encode_jpeg(quality=85)
                assert psnr(np.asarray(Image.open(io.BytesIO(jpeg)).convert("RGB")), rgba[..., :3]) > 28.0
                stream += mjpeg_part(jpeg)
    frames = split_mjpeg(stream)
    assert len(frames) == 3 and all(f[:2] == b"\xff\xd8" for f in frames)
