"""Reader of single-part scanline OpenEXR files (the kind rmd_film_save_exr
and the reference's tinyexr SaveEXR write): FLOAT or HALF channels, stored
uncompressed, ZIPS (one scanline per block) or ZIP (16 per block)."""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

_COMPRESSION = {0: ("none", 1), 2: ("zips", 1), 3: ("zip", 16)}
_PIXEL = {1: np.float16, 2: np.float32}


class ExrError(ValueError):
    pass


def _cstr(b: bytes, at: int) -> tuple[str, int]:
    end = b.index(b"\0", at)
    return b[at:end].decode("latin-1"), end + 1


def read_header(data: bytes) -> tuple[dict, int]:
    """Attributes of the header (channels as a list of (name, pixel type))
    and the offset just after it."""
    if len(data) < 8 or struct.unpack_from("<I", data, 0)[0] != 20000630:
        raise ExrError("not an OpenEXR file")
    version = struct.unpack_from("<I", data, 4)[0]
    if version & 0xff != 2 or version & 0x1e00:  # tiled, long names, deep or multi-part
        raise ExrError(f"unsupported EXR version field {version:#x}")
    at = 8
    header: dict = {}
    while True:
        name, at = _cstr(data, at)
        if name == "":
            return header, at
        typ, at = _cstr(data, at)
        size = struct.unpack_from("<i", data, at)[0]
        at += 4
        value = data[at:at + size]
        at += size
        if typ == "chlist":
            chans, k = [], 0
            while value[k] != 0:
                cname, k = _cstr(value, k)
                ptype = struct.unpack_from("<i", value, k)[0]
                xs, ys = struct.unpack_from("<ii", value, k + 8)
                if (xs, ys) != (1, 1):
                    raise ExrError("subsampled channels are not supported")
                chans.append((cname, ptype))
                k += 16
            header[name] = chans
        elif typ == "compression" or typ == "lineOrder":
            header[name] = value[0]
        elif typ == "box2i":
            header[name] = struct.unpack("<4i", value)
        elif typ == "float":
            header[name] = struct.unpack("<f", value)[0]
        elif typ == "v2f":
            header[name] = struct.unpack("<2f", value)
        else:
            header[name] = value


def _unzip(block: bytes, raw_size: int) -> bytes:
    pre = np.frombuffer(zlib.decompress(block), np.uint8)
    if pre.size != raw_size:
        raise ExrError("ZIP block of the wrong size")
    d = np.cumsum(pre.astype(np.int64) - 128 * (np.arange(pre.size) > 0)) % 256  # undo the deltas
    d = d.astype(np.uint8)
    out = np.empty_like(d)
    half = (raw_size + 1) // 2
    out[0::2] = d[:half]
    out[1::2] = d[half:]
    return out.tobytes()


def read_exr(path: str | Path) -> tuple[dict[str, np.ndarray], dict]:
    """Channels by name as (height, width) float32 arrays, and the header."""
    data = Path(path).read_bytes()
    header, at = read_header(data)
    comp = header.get("compression", 0)
    if comp not in _COMPRESSION:
        raise ExrError(f"unsupported compression {comp}")
    _, lines = _COMPRESSION[comp]
    x0, y0, x1, y1 = header["dataWindow"]
    w, h = x1 - x0 + 1, y1 - y0 + 1
    chans = header["channels"]
    for _, t in chans:
        if t not in _PIXEL:
            raise ExrError(f"unsupported pixel type {t}")
    chunks = (h + lines - 1) // lines
    offsets = struct.unpack_from(f"<{chunks}Q", data, at)
    out = {name: np.zeros((h, w), np.float32) for name, _ in chans}
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        block = data[off + 8:off + 8 + size]
        n = min(lines, y1 + 1 - y)
        raw_size = n * w * sum(np.dtype(_PIXEL[t]).itemsize for _, t in chans)
        if size < raw_size:
            if comp == 0:
                raise ExrError("short uncompressed block")
            block = _unzip(block, raw_size)
        k = 0
        for line in range(n):
            for name, t in chans:
                dt = np.dtype(_PIXEL[t]).newbyteorder("<")
                row = np.frombuffer(block, dt, w, k)
                out[name][y - y0 + line] = row.astype(np.float32)
                k += w * dt.itemsize
    return out, header


def read_rgba(path: str | Path) -> np.ndarray:
    """(height, width, 4) float32 RGBA of an EXR file with R, G, B (and A) channels."""
    ch, _ = read_exr(path)
    a = ch.get("A")
    if a is None:
        a = np.ones_like(ch["R"])
    return np.stack([ch["R"], ch["G"], ch["B"], a], axis=-1)


def write_exr(path: str | Path, img: np.ndarray) -> None:
    """A float image (height, width[, channels]) as an uncompressed FLOAT EXR:
    1 channel as Y, 3 as R, G, B, 4 as R, G, B, A (stored in name order)."""
    a = np.asarray(img, np.float32)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, n = a.shape
    names = {1: ["Y"], 3: ["R", "G", "B"], 4: ["R", "G", "B", "A"]}[n]
    order = sorted(range(n), key=lambda k: names[k])

    def attr(name, typ, value):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(value)) + value

    chl = b"".join(names[k].encode() + b"\0" + struct.pack("<iB3xii", 2, 0, 1, 1) for k in order) + b"\0"
    box = struct.pack("<4i", 0, 0, w - 1, h - 1)
    head = struct.pack("<II", 20000630, 2) + attr("channels", "chlist", chl) + \
        attr("compression", "compression", b"\0") + attr("dataWindow", "box2i", box) + \
        attr("displayWindow", "box2i", box) + attr("lineOrder", "lineOrder", b"\0") + \
        attr("pixelAspectRatio", "float", struct.pack("<f", 1.0)) + \
        attr("screenWindowCenter", "v2f", struct.pack("<2f", 0, 0)) + \
        attr("screenWindowWidth", "float", struct.pack("<f", 1.0)) + b"\0"
    at = len(head) + 8 * h
    table, blocks = [], []
    for y in range(h):
        data = b"".join(a[y, :, k].astype("<f4").tobytes() for k in order)
        table.append(struct.pack("<Q", at))
        blocks.append(struct.pack("<ii", y, len(data)) + data)
        at += 8 + len(data)
    Path(path).write_bytes(head + b"".join(table) + b"".join(blocks))

