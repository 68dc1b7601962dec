"""Gauge-configuration files in the reference's serial binary format.

Layout (reference 4d_Q16/generic/io_lat.c:826-1006, io_lat_utils.c:519-617,
include/io_lat.h:35-57): int32 magic number 20103 (0x4e87), int32 dims[4],
char time_stamp[64], int32 order (0 = natural site order), then a checksum
record {uint32 sum29, uint32 sum31}, then for every site in natural order
(x fastest) NUMLINK = 5 matrices of NCOL x NCOL complex float32.  The
checksums XOR every 32-bit word of the link data rotated left by its running
index mod 29 and mod 31.  Byte-reversed files are recognised by their magic
number.  NCOL is inferred from the file size.

Links are returned as complex128 [5, V, N, N] in lexicographic site order,
the layout of susy_b200.synth; susy_b200.synth.to_ref converts them for
Lattice.set_links.
"""
from __future__ import annotations

import os
import struct
import time

import numpy as np

MAGIC = 20103
HEADER_BYTES = 4 + 16 + 64 + 4
CHECK_BYTES = 8


def checksums(words: np.ndarray):
    """(sum29, sum31) of the uint32 link words, io_lat.c r_serial."""
    w = words.astype(np.uint64)
    idx = np.arange(w.size, dtype=np.uint64)
    out = []
    for m in (29, 31):
        r = idx % np.uint64(m)
        rot = ((w << r) | (w >> (np.uint64(32) - r))) & np.uint64(0xFFFFFFFF)
        out.append(int(np.bitwise_xor.reduce(rot)))
    return out[0], out[1]


def read_gauge(path: str):
    """Return (dims, ncol, links [5, V, N, N] complex128, info dict)."""
    raw = open(path, "rb").read()
    (magic,) = struct.unpack("<i", raw[:4])
    if magic == MAGIC:
        e = "<"
    elif struct.unpack(">i", raw[:4])[0] == MAGIC:
        e = ">"
    else:
        raise ValueError("unrecognised magic number %d in %s" % (magic, path))
    dims = struct.unpack(e + "4i", raw[4:20])
    stamp = raw[20:84].split(b"\0")[0].decode(errors="replace")
    (order,) = struct.unpack(e + "i", raw[84:88])
    V = int(np.prod(dims))
    off = HEADER_BYTES
    if order != 0:
        coords = np.frombuffer(raw, dtype=e + "i4", count=V, offset=off)
        off += 4 * V
    else:
        coords = None
    s29, s31 = struct.unpack(e + "2I", raw[off:off + CHECK_BYTES])
    off += CHECK_BYTES
    nbytes = len(raw) - off
    nn = nbytes // (V * 5 * 8)
    N = int(round(nn ** 0.5))
    if N * N * V * 5 * 8 != nbytes:
        raise ValueError("file size does not match dims %s" % (dims,))
    words = np.frombuffer(raw, dtype=e + "u4", count=V * 5 * N * N * 2, offset=off)
    c29, c31 = checksums(words)
    data = words.view(e + "f4").reshape(V, 5, N, N, 2).astype(np.float64)
    links = data[..., 0] + 1j * data[..., 1]
    if coords is not None:
        full = np.zeros_like(links)
        full[coords] = links
        links = full
    links = np.ascontiguousarray(np.moveaxis(links, 0, 1))
    info = dict(magic=MAGIC, time_stamp=stamp, order=order, sum29=s29, sum31=s31,
                checksum_ok=(c29 == s29 and c31 == s31), byte_reversed=(e == ">"))
    return tuple(dims), N, links, info


def write_gauge(path: str, dims, links: np.ndarray, stamp: str | None = None):
    """Write links [5, V, N, N] in the serial format (save_serial counterpart,
    io_lat.c:377) with natural order, checksums and an ASCII .info file."""
    K, V, N, _ = links.shape
    if K != 5 or V != int(np.prod(dims)):
        raise ValueError("links must be [5, V, N, N] for dims %s" % (dims,))
    a = np.moveaxis(links, 0, 1)
    data = np.stack([a.real, a.imag], axis=-1).astype("<f4")
    words = data.reshape(-1).view("<u4")
    s29, s31 = checksums(words)
    stamp = stamp or time.asctime()
    hdr = struct.pack("<i4i", MAGIC, *dims) + stamp.encode()[:63].ljust(64, b"\0")
    hdr += struct.pack("<i", 0) + struct.pack("<2I", s29, s31)
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(data.tobytes())
    with open(path + ".info", "w") as f:
        f.write('magic_number = %d\ntime_stamp = "%s"\nchecksums = "%x %x"\n'
                % (MAGIC, stamp, s29, s31))
        for k, d in zip("xyzt", dims):
            f.write("n%s = %d\n" % (k, d))
    return s29, s31
