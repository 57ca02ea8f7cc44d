"""PNG images for the image-texture nodes: a reader of the formats the
reference's exporter writes (`_save_image`, materials.py:194-209, saves
textures as PNG or OpenEXR) and a writer used by the tests.

Reader: non-interlaced images of bit depth 8 or 16 (and palette images of
depth 8) in grey, grey + alpha, RGB, RGBA and palette colour types, all five
scanline filters.  Returns (height, width, channels) arrays of uint8 or
uint16: grey as one channel (a single-channel texture), grey + alpha as RGBA,
palette as RGB or RGBA.
"""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

_SIG = b"\x89PNG\r\n\x1a\n"
_CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


class PngError(ValueError):
    pass


def _chunks(data: bytes):
    at = len(_SIG)
    while at + 8 <= len(data):
        n, kind = struct.unpack(">I4s", data[at:at + 8])
        body = data[at + 8:at + 8 + n]
        if len(body) != n:
            raise PngError("truncated chunk")
        yield kind, body
        at += 12 + n
        if kind == b"IEND":
            return
    raise PngError("no IEND chunk")


def _unfilter(raw: np.ndarray, h: int, stride: int, bpp: int) -> np.ndarray:
    rows = raw.reshape(h, stride + 1)
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.uint8)
    for y in range(h):
        f, line = rows[y, 0], rows[y, 1:]
        if f == 0:
            cur = line.copy()
        elif f == 1:  # Sub: cumulative per channel
            cur = np.cumsum(line.reshape(-1, bpp), axis=0, dtype=np.uint8).reshape(-1)
        elif f == 2:  # Up
            cur = line + prev
        elif f in (3, 4):  # Average, Paeth: left-to-right dependency
            cur = np.zeros(stride, np.uint8)
            p16 = prev.astype(np.int16)
            left = np.zeros(bpp, np.int16)
            upleft = np.zeros(bpp, np.int16)
            for x in range(0, stride, bpp):
                up = p16[x:x + bpp]
                if f == 3:
                    pred = (left + up) >> 1
                else:
                    p = left + up - upleft
                    pa, pb, pc = np.abs(p - left), np.abs(p - up), np.abs(p - upleft)
                    pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, up, upleft))
                v = (line[x:x + bpp].astype(np.int16) + pred) & 0xFF
                cur[x:x + bpp] = v
                left, upleft = v, up
        else:
            raise PngError(f"unknown filter type {f}")
        out[y] = cur
        prev = cur
    return out


def read_png(path: str | Path) -> np.ndarray:
    data = Path(path).read_bytes()
    if not data.startswith(_SIG):
        raise PngError("not a PNG file")
    ihdr = None
    palette = trns = None
    idat = []
    for kind, body in _chunks(data):
        if kind == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"PLTE":
            palette = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"tRNS":
            trns = np.frombuffer(body, np.uint8)
        elif kind == b"IDAT":
            idat.append(body)
    if ihdr is None:
        raise PngError("no IHDR chunk")
    w, h, depth, ctype, comp, filt, interlace = ihdr
    if ctype not in _CHANNELS or comp != 0 or filt != 0:
        raise PngError(f"unsupported PNG colour type {ctype}")
    if interlace:
        raise PngError("interlaced PNG is not supported")
    if depth not in (8, 16) or (ctype == 3 and depth != 8):
        raise PngError(f"unsupported PNG bit depth {depth}")
    ch = _CHANNELS[ctype]
    bpp = ch * depth // 8
    raw = np.frombuffer(zlib.decompress(b"".join(idat)), np.uint8)
    if raw.size != h * (w * bpp + 1):
        raise PngError("image data of the wrong size")
    px = _unfilter(raw, h, w * bpp, bpp)
    if depth == 16:
        img = px.reshape(h, w, ch, 2).astype(np.uint16)
        img = (img[..., 0] << 8) | img[..., 1]
    else:
        img = px.reshape(h, w, ch)
    if ctype == 3:
        if palette is None:
            raise PngError("palette image without PLTE")
        idx = img[..., 0]
        rgb = palette[np.minimum(idx, len(palette) - 1)]
        if trns is not None:
            alpha = np.full(256, 255, np.uint8)
            alpha[:len(trns)] = trns
            return np.concatenate([rgb, alpha[idx][..., None]], axis=-1)
        return rgb
    if ctype == 4:  # grey + alpha as RGBA
        g, a = img[..., :1], img[..., 1:]
        return np.concatenate([g, g, g, a], axis=-1)
    return img


def write_png(path: str | Path, img: np.ndarray, filters=(0,)) -> None:
    """An uint8 / uint16 image (h, w[, 1|3|4]) as PNG; rows cycle through `filters`
    (0 none, 1 sub, 2 up, 3 average, 4 Paeth), so tests can exercise each."""
    a = np.asarray(img)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, ch = a.shape
    ctype = {1: 0, 3: 2, 4: 6}[ch]
    depth = 16 if a.dtype == np.uint16 else 8
    if depth == 16:
        px = np.stack([(a >> 8).astype(np.uint8), (a & 0xFF).astype(np.uint8)], axis=-1).reshape(h, -1)
    else:
        px = a.astype(np.uint8).reshape(h, -1)
    bpp = ch * depth // 8
    rows = []
    prev = np.zeros(px.shape[1], np.int16)
    for y in range(h):
        f = filters[y % len(filters)]
        cur = px[y].astype(np.int16)
        left = np.concatenate([np.zeros(bpp, np.int16), cur[:-bpp]])
        upleft = np.concatenate([np.zeros(bpp, np.int16), prev[:-bpp]])
        if f == 0:
            enc = cur
        elif f == 1:
            enc = cur - left
        elif f == 2:
            enc = cur - prev
        elif f == 3:
            enc = cur - ((left + prev) >> 1)
        else:
            p = left + prev - upleft
            pa, pb, pc = np.abs(p - left), np.abs(p - prev), np.abs(p - upleft)
            enc = cur - np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, upleft))
        rows.append(bytes([f]) + (enc & 0xFF).astype(np.uint8).tobytes())
        prev = cur

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    out = _SIG + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 0))
    out += chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b"")
    Path(path).write_bytes(out)
