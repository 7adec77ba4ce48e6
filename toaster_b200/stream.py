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


class AviMjpegWriter:
    """Motion-JPEG video in a RIFF AVI file: one 'vids'/'MJPG' stream whose frames are the JPEG
    bytes given to ``write_frame`` (device-encoded by ``GpuRenderer.encode_jpeg``), with an
    'idx1' key-frame index. Frame counts and sizes are patched into the headers on ``close``.
    The reference writes video by piping RGBA frames to ffmpeg
    (crates/toaster-gpu/src/video_output.rs); this container needs no external encoder."""

    def __init__(self, path, width: int, height: int, fps: int):
        import struct

        if width <= 0 or height <= 0 or fps <= 0:
            raise ValueError("video width, height and fps must be positive")
        self._struct = struct
        self.width, self.height, self.fps = width, height, fps
        self.frames, self.max_size, self._index = 0, 0, []
        self._f = open(path, "wb")
        self._f.write(self._header(0, 0, 0))
        self._movi_start = self._f.tell()
        self._f.write(b"LIST\0\0\0\0movi")

    def _header(self, frames: int, max_size: int, riff_size: int) -> bytes:
        st = self._struct
        avih = st.pack("<10I4I", 1_000_000 // self.fps, max_size * self.fps, 0, 0x10, frames, 0, 1, max_size,
                       self.width, self.height, 0, 0, 0, 0)
        strh = st.pack("<4s4sIHHIIIIIIiI4h", b"vids", b"MJPG", 0, 0, 0, 0, 1, self.fps, 0, frames, max_size, -1, 0,
                       0, 0, self.width, self.height)
        strf = st.pack("<IiiHH4sIiiII", 40, self.width, self.height, 1, 24, b"MJPG", self.width * self.height * 3,
                       0, 0, 0, 0)
        strl = b"strl" + b"strh" + st.pack("<I", len(strh)) + strh + b"strf" + st.pack("<I", len(strf)) + strf
        hdrl = b"hdrl" + b"avih" + st.pack("<I", len(avih)) + avih + b"LIST" + st.pack("<I", len(strl)) + strl
        return b"RIFF" + st.pack("<I", riff_size) + b"AVI " + b"LIST" + st.pack("<I", len(hdrl)) + hdrl

    def write_frame(self, jpeg: bytes) -> None:
        st = self._struct
        jpeg = bytes(jpeg)
        if jpeg[:2] != b"\xff\xd8":
            raise ValueError("not a JPEG frame")
        offset = self._f.tell() - (self._movi_start + 8)  # from the 'movi' fourcc
        self._f.write(b"00dc" + st.pack("<I", len(jpeg)) + jpeg + (b"\0" if len(jpeg) & 1 else b""))
        self._index.append((offset, len(jpeg)))
        self.frames += 1
        self.max_size = max(self.max_size, len(jpeg))

    def close(self) -> None:
        if self._f is None:
            return
        st = self._struct
        end_movi = self._f.tell()
        self._f.write(b"idx1" + st.pack("<I", 16 * len(self._index)))
        for offset, size in self._index:
            self._f.write(b"00dc" + st.pack("<III", 0x10, offset, size))
        end = self._f.tell()
        self._f.seek(0)
        self._f.write(self._header(self.frames, self.max_size, end - 8))
        self._f.seek(self._movi_start + 4)
        self._f.write(st.pack("<I", end_movi - self._movi_start - 8))
        self._f.close()
        self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_avi_mjpeg(path) -> tuple:
    """(width, height, fps, [jpeg frames]) of a file written by AviMjpegWriter, read through its
    'idx1' index (a checker for the writer's layout)."""
    import struct

    data = open(path, "rb").read()
    if data[:4] != b"RIFF" or data[8:12] != b"AVI " or struct.unpack("<I", data[4:8])[0] != len(data) - 8:
        raise ValueError("not a complete RIFF AVI file")
    avih = data.index(b"avih") + 8
    us, _, _, _, frames = struct.unpack("<5I", data[avih:avih + 20])
    width, height = struct.unpack("<2I", data[avih + 32:avih + 40])
    movi = data.index(b"movi")
    idx = data.index(b"idx1", movi)
    n = struct.unpack("<I", data[idx + 4:idx + 8])[0] // 16
    out = []
    for k in range(n):
        ckid, flags, offset, size = struct.unpack("<4sIII", data[idx + 8 + 16 * k:idx + 24 + 16 * k])
        if ckid != b"00dc" or data[movi + offset:movi + offset + 4] != b"00dc":
            raise ValueError("index entry does not point at a frame chunk")
        out.append(data[movi + offset + 8:movi + offset + 8 + size])
    if len(out) != frames:
        raise ValueError("frame count and index disagree")
    return width, height, round(1_000_000 / us), out
