"""TEST INFRASTRUCTURE ONLY -- the oracle's restatement of the reference's reader of Banana
particle data files (.bnn).  Only tests/ use it, to decode the files the CUDA solver's host
class writes exactly as the reference's own tools would.

Restated from:
  ParticleSerialization::read(fileName, readAttributes, bStopIfFailed)
      Simulation/ParticleTools/ParticleSerialization.cpp:643-706
  ParticleSerialization::readHeader(std::ifstream&)          ParticleSerialization.cpp:741-813
  ParticleSerialization::readAttribute                       ParticleSerialization.cpp:816-829
  ParticleSerialization::getFixedAttribute / getParticleAttribute
      ParticleSerialization.cpp:147-160, 212-325
  ParticleHelpers::decompress (vectors, matrices, scalars)
      Simulation/ParticleTools/ParticleHelpers.cpp:183-232, 234-280, 284-320

What the reference reader does, and this restatement keeps:
* The header is read line by line; each line's first whitespace-separated token decides:
  "BananaParticleData" (the magic), "EndHeader." (end), "NParticles n",
  "FixedAttribute|ParticleAttribute name type typeSize count dataSize"; any other token
  makes the read fail.  The file is valid only if the magic was seen.
* Attributes go into two std::map containers (Setup.h:102: Map = std::map), so the data
  blocks are read in the maps' order -- fixed attributes by name (bytewise), then
  particle attributes by name -- whatever order the header lines came in, each block being
  `dataSize` bytes from a running cursor.
* compressed_real vectors of N components: N float minima, N float maxima, then
  nParticles * N uint16; value = q * (max - min) / 65535 + min, evaluated in float as
  ((q * diff) / 65535) + min with diff = max - min.  Matrices: one float minimum and one
  maximum for all N*N entries, the same formula.

Parity status: the reference ships no .bnn files or reader tests for this path, so this
reader is pinned by the restatement alone (parity unpinned by reference fixtures).
"""
from __future__ import annotations

import struct

import numpy as np

_TYPES = {"char", "uint16", "int", "uint", "real", "compressed_real", "vector_char", "vector_int", "vector_uint",
          "vector_real", "vector_compressed_real"}


class BnnReadError(Exception):
    pass


def _read_header(raw: bytes):
    """readHeader(std::ifstream&): returns (nParticles, fixed, particle, data start) or
    raises BnnReadError where the reference returns false."""
    pos = 0
    got_magic = False
    n_particles = 0
    fixed, particle = {}, {}
    while pos < len(raw):
        end = raw.find(b"\n", pos)
        line = raw[pos:] if end < 0 else raw[pos:end]
        pos = len(raw) if end < 0 else end + 1
        toks = line.decode("latin-1").split()
        token = toks[0] if toks else ""
        if token == "BananaParticleData":
            got_magic = True
        elif token == "EndHeader.":
            break
        elif token == "NParticles":
            n_particles = int(toks[1])
        elif token in ("FixedAttribute", "ParticleAttribute"):
            name, type_name, type_size, count, data_size = toks[1], toks[2], int(toks[3]), int(toks[4]), int(toks[5])
            attr = {"name": name, "type": type_name if type_name in _TYPES else "int", "type_size": type_size,
                    "count": count, "data_size": data_size}
            (fixed if token == "FixedAttribute" else particle)[name] = attr
        else:
            raise BnnReadError(f"unknown header line {line!r}")
    if not got_magic:
        raise BnnReadError("no BananaParticleData magic")
    return n_particles, fixed, particle, pos


def read(path):
    """ParticleSerialization::read(fileName) with every attribute: returns
    (nParticles, fixed, particle), each attribute dict carrying its raw `buffer`."""
    raw = open(path, "rb").read()
    n, fixed, particle, cursor = _read_header(raw)
    for table in (fixed, particle):
        for name in sorted(table, key=lambda s: s.encode()):  # std::map<std::string, ...> order
            a = table[name]
            buf = raw[cursor:cursor + a["data_size"]]
            if len(buf) != a["data_size"]:
                raise BnnReadError(f"attribute {name}: file ends inside its data")  # ipf.good() fails
            a["buffer"] = buf
            cursor += a["data_size"]
    return n, fixed, particle


def _plain(a, n_values):
    dt = {"real": np.float32 if a["type_size"] == 4 else np.float64, "uint": np.uint32, "int": np.int32,
          "uint16": np.uint16, "char": np.int8}[a["type"]]
    v = np.frombuffer(a["buffer"], dt)
    if n_values is not None:
        v = v[:n_values]
    return v


def fixed_attribute(fixed, name):
    """getFixedAttribute: the attribute's values (count of them)"""
    a = fixed[name]
    return _plain(a, a["count"])


def _decompress_vectors(buf: bytes, n: int, N: int) -> np.ndarray:
    """ParticleHelpers::decompress(Vec_VecX<N>&, buffer, nParticles) in float"""
    lo = np.frombuffer(buf[:4 * N], np.float32)
    hi = np.frombuffer(buf[4 * N:8 * N], np.float32)
    seg = n * N * 2
    if 8 * N + seg != len(buf):
        raise BnnReadError("compressed vector attribute has the wrong size")
    q = np.frombuffer(buf[8 * N:], np.uint16).reshape(n, N).astype(np.float32)
    diff = (hi - lo).astype(np.float32)
    return ((q * diff) / np.float32(65535.0) + lo).astype(np.float32)


def _decompress_matrices(buf: bytes, n: int, N: int) -> np.ndarray:
    """ParticleHelpers::decompress(Vector<MatXxX<N>>&, buffer, nParticles) in float: the
    N*N entries in glm's column-major memory order"""
    lo, hi = struct.unpack("<ff", buf[:8])
    lo, hi = np.float32(lo), np.float32(hi)
    if 8 + n * N * N * 2 != len(buf):
        raise BnnReadError("compressed matrix attribute has the wrong size")
    q = np.frombuffer(buf[8:], np.uint16).reshape(n, N * N).astype(np.float32)
    diff = np.float32(hi - lo)
    return ((q * diff) / np.float32(65535.0) + lo).astype(np.float32)


def particle_attribute(n, particle, name, matrix_dim: int | None = None):
    """getParticleAttribute: per-particle values, (n, count) (decompressed for
    compressed_real; matrix_dim N reads a compressed N x N matrix attribute)"""
    a = particle[name]
    if a["type"] != "compressed_real":
        return _plain(a, n * a["count"]).reshape(n, a["count"]) if a["count"] > 1 else _plain(a, n)
    if matrix_dim is not None:
        if matrix_dim * matrix_dim != a["count"]:
            raise BnnReadError("matrix dimension does not match the attribute count")
        return _decompress_matrices(a["buffer"], n, matrix_dim)
    return _decompress_vectors(a["buffer"], n, a["count"])
