"""Oracle (test infrastructure): restatement of the reference's Gadget-1
reader, load_particles (src/load.cpp:34-96), and a writer of such files for
the tests (io_header_1 layout, tigergrav/load.hpp:20-39)."""
import struct

import numpy as np

HEADER = struct.Struct("<6I6dddii6Iiiddddiii84x")
assert HEADER.size == 256


def write(path, pos, vel, redshift=49.0, mass=1.0, omega_m=0.3, omega_lambda=0.7, h=0.7, box=1.0):
    n = len(pos)
    hdr = HEADER.pack(0, n, 0, 0, 0, 0, 0.0, mass, 0.0, 0.0, 0.0, 0.0, 1.0 / (1.0 + redshift), redshift, 0, 0,
                      0, n, 0, 0, 0, 0, 0, 1, box, omega_m, omega_lambda, h, 0, 0, 0)
    with open(path, "wb") as f:
        for block in (hdr, np.ascontiguousarray(pos, "<f4").tobytes(), np.ascontiguousarray(vel, "<f4").tobytes()):
            f.write(struct.pack("<i", len(block)))
            f.write(block)
            f.write(struct.pack("<i", len(block)))


def _double_to_pos(x):
    """tigergrav/position.hpp:30-37: lround((x - 0.5) 2^32), wrapped (lround: ties away from zero)"""
    y = (np.asarray(x, np.float64) - 0.5) * 4294967296.0
    z = np.where(y >= 0, np.floor(y + 0.5), np.ceil(y - 0.5))
    z = np.where(z >= 2147483648.0, z - 4294967296.0, z)
    return z.astype(np.int64).astype(np.int32)


def load(path):
    with open(path, "rb") as f:
        buf = f.read()
    h = HEADER.unpack_from(buf, 4)
    n = h[1]
    redshift = h[13]
    off = 4 + 256 + 4 + 4
    pos = np.frombuffer(buf, "<f4", 3 * n, off).reshape(n, 3).copy()
    off += 12 * n + 4 + 4
    vel = np.frombuffer(buf, "<f4", 3 * n, off).reshape(n, 3)
    sep = 0.5 * float(n) ** (-1.0 / 3.0)
    p = (pos.astype(np.float64) + sep).astype(np.float32)      # float += double
    for _ in range(4):                                        # while (x > 1) x -= 1, in float
        p = np.where(p > 1.0, (p.astype(np.float64) - 1.0).astype(np.float32), p)
    x = _double_to_pos(p.astype(np.float64))
    c0 = 1.0 / (1.0 + redshift)
    v = (vel.astype(np.float64) * c0 ** 1.5).astype(np.float32)
    return n, x, v
