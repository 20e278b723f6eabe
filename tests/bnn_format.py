"""Reader of Banana particle data files (.bnn) for the tests: text header
(FixedAttribute / ParticleAttribute lines, NParticles, EndHeader.) then the attribute
blobs in header order; compressed_real = float min[c], float max[c], uint16 per value
(a matrix attribute: one float min and one float max for all its entries)."""
import numpy as np


def read_bnn(path):
    raw = open(path, "rb").read()
    lines, pos = [], 0
    while True:
        end = raw.index(b"\n", pos)
        line = raw[pos:end].decode()
        pos = end + 1
        lines.append(line)
        if line == "EndHeader.":
            break
    assert lines[0] == "BananaParticleData"
    attrs, order, n = {}, [], None
    for line in lines[1:-1]:
        f = line.split()
        if f[0] == "NParticles":
            n = int(f[1])
            continue
        assert f[0] in ("FixedAttribute", "ParticleAttribute")
        name, typ, esize, count, nbytes = f[1], f[2], int(f[3]), int(f[4]), int(f[5])
        attrs[name] = {"kind": f[0], "type": typ, "esize": esize, "count": count, "bytes": nbytes}
        order.append(name)
    for name in order:
        a = attrs[name]
        a["raw"] = raw[pos:pos + a["bytes"]]
        pos += a["bytes"]
    assert pos == len(raw)
    return n, attrs, order


def values(attr):
    """numpy values of an attribute (decoded for compressed_real)"""
    t, c, b = attr["type"], attr["count"], attr["raw"]
    if t == "real":
        return np.frombuffer(b, np.float32)
    if t == "uint":
        return np.frombuffer(b, np.uint32)
    if t == "uint16":
        return np.frombuffer(b, np.uint16)
    if t == "compressed_real":
        lo = np.frombuffer(b[:4 * c], np.float32)
        hi = np.frombuffer(b[4 * c:8 * c], np.float32)
        q = np.frombuffer(b[8 * c:], np.uint16).reshape(-1, c).astype(np.float32)
        return q * (hi - lo) / np.float32(65535.0) + lo, lo, hi, q
    raise ValueError(t)


def matrix_values(attr):
    """decoded matrix attribute (compressed_real with one min / max for all entries)"""
    c, b = attr["count"], attr["raw"]
    assert attr["type"] == "compressed_real"
    lo, hi = np.frombuffer(b[:8], np.float32)
    q = np.frombuffer(b[8:], np.uint16).reshape(-1, c).astype(np.float32)
    return q * (hi - lo) / np.float32(65535.0) + lo, lo, hi, q
