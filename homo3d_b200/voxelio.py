"""Density files in the reference's binary voxel format (homo::binary,
homogenization/grid.cpp:471-485 writeDensity, :578-597 readDensity): three int32
cell counts (x, y, z) followed by one float32 per cell in lexicographic order,
x fastest, little-endian.  The OpenVDB format of the reference needs the OpenVDB
library and is not provided.

    rho, reso = read_density("rho.bin")
    write_density("rho.bin", rho, reso)
"""
import numpy as np


def write_density(path, rho, reso):
    """rho: cell values in lexicographic order (any array of prod(reso) values)"""
    reso = tuple(int(r) for r in reso)
    a = np.ascontiguousarray(np.asarray(rho, dtype="<f4").reshape(-1))
    if a.size != reso[0] * reso[1] * reso[2]:
        raise ValueError("density has %d values, the resolution %r needs %d" % (a.size, reso, np.prod(reso)))
    with open(path, "wb") as f:
        f.write(np.asarray(reso, dtype="<i4").tobytes())
        f.write(a.tobytes())


def read_density(path):
    """(rho float32 [prod(reso)] lexicographic, reso (x, y, z)); a short file raises"""
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(12), dtype="<i4")
        if head.size != 3 or np.any(head <= 0):
            raise ValueError("%s: not a binary density file" % path)
        reso = tuple(int(v) for v in head)
        n = reso[0] * reso[1] * reso[2]
        rho = np.frombuffer(f.read(4 * n), dtype="<f4")
    if rho.size != n:
        raise ValueError("%s: file is not complete (%d of %d values)" % (path, rho.size, n))
    return rho.astype(np.float32), reso
