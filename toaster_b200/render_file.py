"""Renders a toaster scene file on the GPU and writes the displayed image.

    python -m toaster_b200.render_file scene.json -o frame.png [--spp N] [--frame F] [--guiding]

The CUDA counterpart of ``toaster-cli gpu-render`` (crates/toaster-cli/src/main.rs:267-330): the
scene is loaded and packed by the library's native loader (tc_scene_load), uploaded, rendered,
display-converted on the device with the scene's exposure (ACES, sRGB, RGBA8) and written as PNG,
or JPEG-encoded on the device when the output ends in .jpg / .jpeg. Prints one JSON line with
the timings.
"""

from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

from .renderer import GpuRenderer
from .stream import encode_png


def render_file(scene: Path, output: Path, spp: int = 0, frame: int = 0, guiding: bool = False, device: int = 0,
                quality: int = 90) -> dict:
    """Loads, renders and writes one scene file; returns timings and sizes."""
    t0 = time.perf_counter()
    with GpuRenderer(device) as r:
        exposure = r.upload_file(scene)
        t1 = time.perf_counter()
        r.render(samples=spp or None, frame_index=frame, guiding=guiding)
        stats = r.stats()
        if output.suffix.lower() in (".jpg", ".jpeg"):
            data = r.encode_jpeg(quality, exposure)
        else:
            data = encode_png(r.readback_rgba8(exposure))
        output.write_bytes(data)
        t2 = time.perf_counter()
        return {"scene": str(scene), "output": str(output), "width": r.width, "height": r.height,
                "samples": stats.get("paths", 0) // max(1, r.width * r.height), "exposure_stops": exposure,
                "load_upload_ms": (t1 - t0) * 1e3, "kernel_ms": stats.get("kernel_ms"),
                "total_ms": (t2 - t0) * 1e3, "bytes": len(data)}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("scene", type=Path)
    ap.add_argument("-o", "--output", type=Path, required=True)
    ap.add_argument("--spp", type=int, default=0, help="samples per pixel (default: the scene's)")
    ap.add_argument("--frame", type=int, default=0)
    ap.add_argument("--guiding", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--quality", type=int, default=90)
    a = ap.parse_args()
    print(json.dumps(render_file(a.scene, a.output, a.spp, a.frame, a.guiding, a.device, a.quality)))


if __name__ == "__main__":
    main()
