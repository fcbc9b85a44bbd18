"""Minimal single-band GeoTIFF read/write in numpy (no GDAL).

The reference exchanges rasters as GeoTIFF through GDAL (GeoTIFF.cpp:20-577):
masks in (any band type, returned as float, row 0 at the top, geotransform
and NoData value), Float32 density out.  This module covers that layout for
Python callers and tests: uncompressed strips or tiles, classic TIFF or
BigTIFF, 8/16/32-bit integer and 32/64-bit float samples.  The C++ host driver
has the same codec in csrc/tiff_io.hpp (which also reads LZW).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

_TYPE_SIZE = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 1, 7: 1, 8: 2, 9: 4, 10: 8, 11: 4, 12: 8, 16: 8, 17: 8, 18: 8}


@dataclass
class GeoRaster:
    """Band 1 of a GeoTIFF: data[row, col] with row 0 at the top."""

    data: np.ndarray
    geotransform: tuple = (0.0, 1.0, 0.0, 0.0, 0.0, -1.0)
    nodata: float | None = None
    block: tuple = field(default=(0, 0))

    @property
    def xll(self) -> float:
        return self.geotransform[0]

    @property
    def yll(self) -> float:
        return self.geotransform[3] + self.data.shape[0] * self.geotransform[5]

    @property
    def cell_size(self) -> float:
        return self.geotransform[1]


def read(path: str) -> GeoRaster:
    buf = open(path, "rb").read()
    bo = {b"II": "<", b"MM": ">"}.get(buf[:2])
    if bo is None:
        raise ValueError(f"{path}: not a TIFF")
    magic = struct.unpack(bo + "H", buf[2:4])[0]
    big = magic == 43
    if magic not in (42, 43):
        raise ValueError(f"{path}: bad magic {magic}")
    ifd = struct.unpack(bo + ("Q" if big else "I"), buf[8:16] if big else buf[4:8])[0]
    n = struct.unpack(bo + ("Q" if big else "H"), buf[ifd: ifd + (8 if big else 2)])[0]
    esz, base = (20, ifd + 8) if big else (12, ifd + 2)
    tags = {}
    for i in range(n):
        e = buf[base + i * esz: base + (i + 1) * esz]
        tag, typ = struct.unpack(bo + "HH", e[:4])
        cnt = struct.unpack(bo + ("Q" if big else "I"), e[4:12] if big else e[4:8])[0]
        size = _TYPE_SIZE.get(typ, 1) * cnt
        inline = 8 if big else 4
        raw = e[12:12 + size] if big and size <= inline else (e[8:8 + size] if size <= inline else None)
        if raw is None:
            off = struct.unpack(bo + ("Q" if big else "I"), e[12:20] if big else e[8:12])[0]
            raw = buf[off: off + size]
        if typ == 2:
            val = raw.rstrip(b"\0").decode("latin1")
        elif typ == 12:
            val = struct.unpack(bo + f"{cnt}d", raw)
        else:
            code = {1: "B", 3: "H", 4: "I", 16: "Q", 8: "h", 9: "i", 6: "b"}.get(typ, "B")
            val = struct.unpack(bo + f"{cnt}{code}", raw)
        tags[tag] = val
    ncols, nrows = tags[256][0], tags[257][0]
    bits = tags.get(258, (8,))[0]
    fmt = tags.get(339, (1,))[0]
    if tags.get(259, (1,))[0] != 1:
        raise ValueError(f"{path}: compressed TIFFs are read by the C++ codec only")
    dt = np.dtype({(3, 32): "f4", (3, 64): "f8", (1, 8): "u1", (1, 16): "u2", (1, 32): "u4",
                   (2, 8): "i1", (2, 16): "i2", (2, 32): "i4"}[(fmt, bits)]).newbyteorder(bo)
    out = np.zeros((nrows, ncols), np.float32)
    if 322 in tags:
        bw, bh = tags[322][0], tags[323][0]
        offs, cnts = tags[324], tags[325]
        nbx = (ncols + bw - 1) // bw
        for k, (o, c) in enumerate(zip(offs, cnts)):
            by, bx = divmod(k, nbx)
            blk = np.frombuffer(buf[o: o + bw * bh * dt.itemsize], dt).reshape(bh, bw)
            rr, cc = min(bh, nrows - by * bh), min(bw, ncols - bx * bw)
            out[by * bh: by * bh + rr, bx * bw: bx * bw + cc] = blk[:rr, :cc]
    else:
        bw, bh = ncols, tags.get(278, (nrows,))[0]
        row = 0
        for o, c in zip(tags[273], tags[279]):
            rr = min(bh, nrows - row)
            out[row: row + rr] = np.frombuffer(buf[o: o + rr * ncols * dt.itemsize], dt).reshape(rr, ncols)
            row += rr
    gt = (0.0, 1.0, 0.0, 0.0, 0.0, -1.0)
    if 33550 in tags and 33922 in tags:
        sx, sy = tags[33550][0], tags[33550][1]
        t = tags[33922]
        gt = (t[3] - t[0] * sx, sx, 0.0, t[4] + t[1] * sy, 0.0, -sy)
    nd = float(tags[42113]) if 42113 in tags else None
    return GeoRaster(out, gt, nd, (bw, bh))


def write(path: str, r: GeoRaster) -> None:
    """Writes a Float32, uncompressed, single-strip GeoTIFF."""
    data = np.ascontiguousarray(r.data, dtype="<f4")
    nrows, ncols = data.shape
    gt = r.geotransform
    payload = bytearray()
    entries = []

    def add(tag, typ, cnt, value_bytes):
        entries.append((tag, typ, cnt, bytes(value_bytes)))

    add(256, 4, 1, struct.pack("<I", ncols))
    add(257, 4, 1, struct.pack("<I", nrows))
    add(258, 3, 1, struct.pack("<H", 32))
    add(259, 3, 1, struct.pack("<H", 1))
    add(262, 3, 1, struct.pack("<H", 1))
    add(273, 4, 1, b"")  # patched
    add(277, 3, 1, struct.pack("<H", 1))
    add(278, 4, 1, struct.pack("<I", nrows))
    add(279, 4, 1, struct.pack("<I", data.nbytes))
    add(339, 3, 1, struct.pack("<H", 3))
    add(33550, 12, 3, struct.pack("<3d", gt[1], -gt[5], 0.0))
    add(33922, 12, 6, struct.pack("<6d", 0.0, 0.0, 0.0, gt[0], gt[3], 0.0))
    if r.nodata is not None:
        s = (repr(float(r.nodata)).rstrip("0").rstrip(".") if float(r.nodata) != int(r.nodata)
             else str(int(r.nodata))).encode() + b"\0"
        add(42113, 2, len(s), s)
    entries.sort()
    header = 8
    ifd_size = 2 + 12 * len(entries) + 4
    pay_off = header + ifd_size
    blobs = {}
    for tag, typ, cnt, vb in entries:
        if len(vb) > 4:
            blobs[tag] = pay_off + len(payload)
            payload += vb
            if len(payload) % 2:
                payload += b"\0"
    data_off = pay_off + len(payload)
    out = bytearray(b"II*\0" + struct.pack("<I", header))
    out += struct.pack("<H", len(entries))
    for tag, typ, cnt, vb in entries:
        if tag == 273:
            vb = struct.pack("<I", data_off)
        out += struct.pack("<HHI", tag, typ, cnt)
        out += struct.pack("<I", blobs[tag]) if tag in blobs else vb.ljust(4, b"\0")
    out += struct.pack("<I", 0)
    out += payload
    out += data.tobytes()
    with open(path, "wb") as f:
        f.write(out)
