"""MJPEG frames for live previews, fed from the device.

The reference's preview server (crates/toaster-server/src/routes.rs:82-110) streams
``multipart/x-mixed-replace; boundary=frame`` parts, one JPEG per rendered frame, each JPEG made
on the host by ``encode_pixels_to_jpeg`` (crates/toaster-gpu/src/image_output.rs:27-56) after a
float4 readback. Here the frame is display-converted and JPEG-encoded on the device
(``GpuRenderer.encode_jpeg``); only the compressed bytes leave the GPU. The HTTP server itself is
not part of this package: ``mjpeg_part`` builds the same parts for any server or file.
"""

from __future__ import annotations

from typing import BinaryIO, Iterable

MJPEG_BOUNDARY = "frame"
CONTENT_TYPE = f"multipart/x-mixed-replace; boundary={MJPEG_BOUNDARY}"


def mjpeg_part(jpeg: bytes) -> bytes:
    """One JPEG wrapped in a complete multipart part: boundary, headers, body, trailing CRLF."""
    header = f"--{MJPEG_BOUNDARY}\r\nContent-Type: image/jpeg\r\nContent-Length: {len(jpeg)}\r\n\r\n"
    return header.encode("ascii") + bytes(jpeg) + b"\r\n"


def split_mjpeg(stream: bytes) -> list:
    """The JPEG bodies of a stream of parts (inverse of concatenated ``mjpeg_part`` calls)."""
    out, pos = [], 0
    marker = f"--{MJPEG_BOUNDARY}\r\n".encode("ascii")
    while pos < len(stream):
        if not stream.startswith(marker, pos):
            raise ValueError(f"no boundary at byte {pos}")
        head_end = stream.index(b"\r\n\r\n", pos)
        headers = stream[pos + len(marker):head_end].decode("ascii").split("\r\n")
        length = next(int(h.split(":", 1)[1]) for h in headers if h.lower().startswith("content-length"))
        body = head_end + 4
        out.append(stream[body:body + length])
        pos = body + length + 2
    return out


def write_mjpeg(frames: Iterable[bytes], sink: BinaryIO) -> int:
    """Writes JPEG frames as MJPEG parts; returns the number written."""
    n = 0
    for jpeg in frames:
        sink.write(mjpeg_part(jpeg))
        n += 1
    return n


def encode_png(rgba) -> bytes:
    """An (height, width, 4) uint8 image as a PNG file (8-bit RGBA, filter type 0), the format
    the reference's ``save_png`` writes (crates/toaster-gpu/src/image_output.rs:59)."""
    import struct
    import zlib

    import numpy as np

    img = np.ascontiguousarray(rgba, np.uint8)
    h, w, c = img.shape
    if c != 4:
        raise ValueError("expected an RGBA image")
    rows = np.concatenate([np.zeros((h, 1), np.uint8), img.reshape(h, w * 4)], axis=1)

    def chunk(kind: bytes, body: bytes) -> bytes:
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(rows.tobytes(), 6)) + chunk(b"IEND", b""))
