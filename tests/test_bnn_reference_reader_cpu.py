"""The .bnn files the C++ host class writes, decoded by the restatement of the reference's
own reader (oracle/bnn_reader.py: ParticleSerialization::read / readHeader /
readAttribute and ParticleHelpers::decompress), not by this repository's reader."""
import struct
import subprocess

import numpy as np
import pytest

from banana_b200 import build as bld
from oracle import bnn_reader as R
from tests.test_host_cpu import BNN_SELFTEST


@pytest.fixture(scope="module")
def selftest_file(tmp_path_factory):
    d = tmp_path_factory.mktemp("bnn")
    src = d / "t.cpp"
    src.write_text(BNN_SELFTEST)
    exe = d / "t"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(bld.HOST), str(src), str(bld.HOST / "bnn_io.cpp"), "-o",
                    str(exe)], check=True)
    out = d / "f.bnn"
    subprocess.run([str(exe), str(out)], check=True)
    return out


def test_reference_reader_decodes_written_file(selftest_file):
    n, fixed, particle = R.read(selftest_file)
    assert n == 5
    assert R.fixed_attribute(fixed, "particle_radius")[0] == np.float32(0.25)
    assert list(R.fixed_attribute(fixed, "grid_resolution")) == [7, 8, 9]
    assert list(R.fixed_attribute(fixed, "NObjects")) == [2]
    src = np.array([0, 1, 2, .5, -1, 2.5, .25, 0, 2, 1, 1, 3, .75, .5, 2.25], np.float32).reshape(5, 3)
    assert np.array_equal(R.particle_attribute(n, particle, "particle_velocity"), src)
    pos = R.particle_attribute(n, particle, "particle_position")
    rng = src.max(0) - src.min(0)
    assert np.all(np.abs(pos - src) <= rng / 65535 + 1e-6)
    assert list(R.particle_attribute(n, particle, "object_index")) == [0, 1, 1, 0, 1]
    mats = ((np.arange(45) * 7) % 13).astype(np.float32) * np.float32(0.1) - np.float32(0.3)
    K = R.particle_attribute(n, particle, "anisotropic_kernel", matrix_dim=3)
    assert K.shape == (5, 9)
    assert np.abs(K.reshape(-1) - mats).max() <= (mats.max() - mats.min()) / 65535 * 1.01


def _file(header_lines, blocks):
    return ("\n".join(header_lines) + "\n").encode() + b"".join(blocks)


def test_reader_takes_data_blocks_in_map_order(tmp_path):
    """The reference reads the data blocks in std::map order (fixed attributes by name, then
    particle attributes by name), not in the order of the header lines."""
    a = struct.pack("<f", 1.5)
    b = struct.pack("<3I", 4, 5, 6)
    p = tmp_path / "x.bnn"
    # header lists b_attr before a_attr; the blocks are in name order (a, then b)
    p.write_bytes(_file(["BananaParticleData", "FixedAttribute b_attr uint 4 3 12", "FixedAttribute a_attr real 4 1 4",
                         "NParticles 0", "EndHeader."], [a, b]))
    n, fixed, _ = R.read(p)
    assert R.fixed_attribute(fixed, "a_attr")[0] == np.float32(1.5)
    assert list(R.fixed_attribute(fixed, "b_attr")) == [4, 5, 6]


def test_reader_refuses_what_the_reference_refuses(tmp_path):
    p = tmp_path / "bad.bnn"
    p.write_bytes(_file(["BananaParticleData", "Something else", "EndHeader."], []))
    with pytest.raises(R.BnnReadError):
        R.read(p)
    p.write_bytes(_file(["NParticles 0", "EndHeader."], []))
    with pytest.raises(R.BnnReadError):
        R.read(p)
