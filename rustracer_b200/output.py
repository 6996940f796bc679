"""Writing developed frames: the reference's save_png (output.rs:113-150) over
the device develop step (apply_optics + tone_map, rt_develop).  PNG encoding
is the standard one (signature, IHDR, one zlib IDAT of filter-0 rows, IEND),
written with the standard library."""
import os
import struct
import zlib

import numpy as np


def write_png(path, rgb8):
    """Write an (H, W, 3) uint8 image as an 8-bit RGB PNG."""
    rgb8 = np.ascontiguousarray(rgb8, np.uint8)
    if rgb8.ndim != 3 or rgb8.shape[2] != 3:
        raise ValueError("expected an (H, W, 3) uint8 image")
    h, w = rgb8.shape[:2]

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    raw = np.concatenate([np.zeros((h, 1), np.uint8), rgb8.reshape(h, w * 3)], axis=1).tobytes()
    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) + \
        chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as fh:
        fh.write(png)
    return path


def read_png(path):
    """Read back an 8-bit RGB PNG written by write_png (filter type 0 rows)."""
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n, tag = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        if zlib.crc32(tag + body) & 0xFFFFFFFF != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError("bad PNG chunk CRC")
        if tag == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            if depth != 8 or ctype != 2:
                raise ValueError("only 8-bit RGB PNGs")
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    rows = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * 3)
    if rows[:, 0].any():
        raise ValueError("only unfiltered rows")
    return rows[:, 1:].reshape(h, w, 3).copy()


def png_name(scene_name, spp):
    """save_png's default file name (output.rs:133-136): render_<slug>_<spp:04>spp.png."""
    return f"render_{scene_name.lower().replace(' ', '_')}_{int(spp):04d}spp.png"


def save_png(gpu_scene, width, height, scene_name, spp, linear=None, exposure=1.0, tonemapper="agx", vignette=0.0,
             distortion=0.0, path=None):
    """Develop the scene's accumulators (or a linear image) on the device and
    write the PNG (main.rs:571-583, output.rs:113-150).  Returns the path."""
    rgb8 = gpu_scene.develop(width, height, linear=linear, exposure=exposure, tonemapper=tonemapper,
                             vignette=vignette, distortion=distortion)
    if not isinstance(rgb8, np.ndarray):
        rgb8 = rgb8.cpu().numpy()
    path = path or png_name(scene_name, spp)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    return write_png(path, rgb8)
