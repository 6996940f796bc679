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
    """Decode a non-interlaced PNG (grey, RGB, palette, grey+alpha, RGBA; 8 or
    16 bits; filter types 0-4) into an (H, W, 3) uint8 RGB image (16-bit
    samples keep their high byte, alpha is dropped) — what `image::open(..)
    .into_rgb8()` gives the reference's textures (texture.rs:21-23)."""
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError(f"{path}: not a PNG file")
    pos, idat, palette, hdr = 8, [], None, None
    while pos < len(data):
        n, tag = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        if zlib.crc32(tag + body) & 0xFFFFFFFF != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError(f"{path}: bad PNG chunk CRC")
        if tag == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"PLTE":
            palette = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif tag == b"IDAT":
            idat.append(body)
        elif tag == b"IEND":
            break
        pos += 12 + n
    w, h, depth, ctype, _, _, interlace = hdr
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}.get(ctype)
    if channels is None or depth not in (8, 16) or interlace or (ctype == 3 and depth != 8):
        raise ValueError(f"{path}: unsupported PNG (colour type {ctype}, depth {depth}, interlace {interlace})")
    bpp = channels * depth // 8
    stride = w * bpp
    raw = np.frombuffer(zlib.decompress(b"".join(idat)), np.uint8).reshape(h, 1 + stride)
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        ft, line = raw[y, 0], raw[y, 1:].astype(np.int32)
        cur = np.zeros(stride, np.int32)
        if ft == 0:
            cur = line
        elif ft == 1:
            for i in range(stride):
                cur[i] = (line[i] + (cur[i - bpp] if i >= bpp else 0)) & 0xFF
        elif ft == 2:
            cur = (line + prev) & 0xFF
        elif ft == 3:
            for i in range(stride):
                cur[i] = (line[i] + ((cur[i - bpp] if i >= bpp else 0) + prev[i]) // 2) & 0xFF
        elif ft == 4:
            for i in range(stride):
                a = cur[i - bpp] if i >= bpp else 0
                b, c = prev[i], (prev[i - bpp] if i >= bpp else 0)
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pred = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cur[i] = (line[i] + pred) & 0xFF
        else:
            raise ValueError(f"{path}: bad PNG filter {ft}")
        out[y] = cur
        prev = cur
    px = out.reshape(h, w, bpp)
    if depth == 16:
        px = px[..., 0::2]                         # high byte of each big-endian sample
    if ctype == 3:
        return palette[px[..., 0]].copy()
    if ctype in (0, 4):
        return np.repeat(px[..., :1], 3, axis=2).copy()
    return px[..., :3].copy()


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
