"""The C++ host side without a GPU: the scene reader and the seeded particle sampler of
FLIP_GPU_Solver produce exactly the particles of banana_b200.scenes.dam_break."""
import subprocess

import numpy as np
import pytest

from banana_b200 import build as bld
from banana_b200 import scenes
from tests.bnn_format import matrix_values, read_bnn, values
from tests.host_scene import dam_break_scene, read_particles


@pytest.fixture(scope="module")
def driver():
    if not bld.LIB.exists():
        bld.build_cuda()
    exe = bld.build_host()
    assert exe is not None and exe.exists()
    return exe


@pytest.mark.parametrize("n", [24, 64])
def test_scene_sampler_matches_python_seeder(driver, tmp_path, n):
    scene = tmp_path / "dam.json"
    scene.write_text(dam_break_scene(n))
    out = tmp_path / "p.f32"
    subprocess.run([str(driver), str(scene), "--sample-only", str(out)], check=True, timeout=60)
    pos, vel = read_particles(out)
    pp, vv = scenes.dam_break(n)
    assert np.array_equal(pos, pp)
    assert np.array_equal(vel, vv)


def test_unknown_solver_is_refused(driver, tmp_path):
    scene = tmp_path / "x.json"
    scene.write_text(dam_break_scene(16, solver="SPH_3DSolver"))
    r = subprocess.run([str(driver), str(scene)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "not supported" in r.stderr


BNN_SELFTEST = r"""
#include "bnn_io.h"
#include <cstdio>
#include <vector>
int main(int argc, char** argv) {
    bnnhost::BnnFile f;
    f.nParticles = 5;
    const float radius = 0.25f;
    const unsigned res[3] = {7, 8, 9};
    const unsigned nobj = 2;
    std::vector<float> pos = {0.f, 1.f, 2.f, 0.5f, -1.f, 2.5f, 0.25f, 0.f, 2.f, 1.f, 1.f, 3.f, 0.75f, 0.5f, 2.25f};
    std::vector<unsigned short> idx = {0, 1, 1, 0, 1};
    f.setFixedReal("particle_radius", &radius, 1);
    f.setFixedUInt("grid_resolution", res, 3);
    f.setFixedUInt("NObjects", &nobj, 1);
    f.setParticleReal("particle_velocity", pos.data(), 3);
    f.setParticleCompressed("particle_position", pos.data(), 3);
    f.setParticleUInt16("object_index", idx.data());
    std::vector<float> mats(45);
    for(int i = 0; i < 45; ++i) mats[i] = 0.1f * (float)((i * 7) % 13) - 0.3f;
    f.setParticleCompressedMatrix("anisotropic_kernel", mats.data(), 3);
    if(!f.write(argv[1])) return 1;
    bnnhost::BnnFile g;
    if(!g.read(argv[1])) return 2;
    std::vector<float> v, c;
    std::vector<unsigned> u;
    if(!g.getFloats("particle_velocity", v) || v != pos) return 3;
    if(!g.getUInts("grid_resolution", u) || u.size() != 3 || u[2] != 9) return 4;
    if(!g.getFloats("particle_position", c) || c.size() != pos.size()) return 5;
    for(size_t i = 0; i < c.size(); ++i) if(c[i] < pos[i] - 1e-4f || c[i] > pos[i] + 1e-4f) return 6;
    std::vector<float> m;
    if(!g.getMatrixFloats("anisotropic_kernel", m) || m.size() != 45) return 7;
    for(size_t i = 0; i < m.size(); ++i) if(m[i] < mats[i] - 2e-5f || m[i] > mats[i] + 2e-5f) return 8;
    return 0;
}
"""


def test_bnn_file_format_round_trip(tmp_path):
    """The .bnn writer / reader of the C++ class: the reference's header layout, attribute
    order (fixed, then particle, each by name), raw and 16-bit compressed encodings."""
    src = tmp_path / "t.cpp"
    src.write_text(BNN_SELFTEST)
    exe = tmp_path / "t"
    host = bld.HOST
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(host), str(src), str(host / "bnn_io.cpp"), "-o", str(exe)],
                   check=True)
    out = tmp_path / "f.bnn"
    subprocess.run([str(exe), str(out)], check=True)
    n, attrs, order = read_bnn(out)
    assert n == 5
    assert order == ["NObjects", "grid_resolution", "particle_radius", "anisotropic_kernel", "object_index",
                     "particle_position", "particle_velocity"]
    assert attrs["particle_radius"]["type"] == "real" and attrs["particle_radius"]["bytes"] == 4
    assert list(values(attrs["grid_resolution"])) == [7, 8, 9]
    pos = values(attrs["particle_velocity"]).reshape(5, 3)
    dec, lo, hi, q = values(attrs["particle_position"])
    assert attrs["particle_position"]["bytes"] == 24 + 2 * 15
    assert np.array_equal(lo, pos.min(0)) and np.array_equal(hi, pos.max(0))
    expect = np.trunc(np.float32(65535.0) * ((pos - lo) / np.where(hi > lo, hi - lo, 1))).astype(np.uint16)
    assert np.array_equal(q.astype(np.uint16), expect)
    assert np.abs(dec - pos).max() <= (hi - lo).max() / 65535 + 1e-6
    assert list(values(attrs["object_index"])) == [0, 1, 1, 0, 1]
    # matrices: one range for all entries (ParticleHelpers.cpp:82-114)
    mats = ((np.arange(45) * 7) % 13).astype(np.float32) * np.float32(0.1) - np.float32(0.3)
    K, klo, khi, kq = matrix_values(attrs["anisotropic_kernel"])
    assert attrs["anisotropic_kernel"]["count"] == 9 and attrs["anisotropic_kernel"]["bytes"] == 8 + 2 * 45
    assert klo == mats.min() and khi == mats.max()
    assert np.array_equal(kq.reshape(-1).astype(np.uint16),
                          np.trunc(np.float32(65535.0) * ((mats - klo) / (khi - klo))).astype(np.uint16))
    assert np.abs(K.reshape(-1) - mats).max() <= (khi - klo) / 65535 * 1.01


ANIM_SELFTEST = r"""
#include "boundary_objects.h"
#include "json_lite.h"
#include <cstdio>
#include <fstream>
#include <sstream>
int main(int argc, char** argv) {
    std::ifstream f(argv[1]);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    bnnhost::Json j = bnnhost::JsonParser(text).parse();
    std::string err;
    auto objs = bnnhost::parse_boundary_objects(j, err);
    if(!err.empty()) { std::printf("error %s\n", err.c_str()); return 0; }
    auto dump = [&](const char* tag, double x) {
        for(const auto& b : objs) {
            std::printf("%s %.6f %d %d", tag, x, b.current.transformed, b.current.dynamic);
            for(int q = 0; q < 12; ++q) std::printf(" %.9g", b.current.inv_transform[q]);
            std::printf(" %.9g\n", b.current.uniform_scale);
        }
    };
    dump("init", 0.0);
    const double times[][2] = {{1, 0.0}, {1, 0.5}, {2, 0.25}, {4, 0.0}, {6, 0.75}, {9, 0.0}};
    for(const auto& t : times) {
        for(auto& b : objs) if(b.dynamic) b.update((unsigned)t[0], t[1]);
        dump("t", t[0] + t[1]);
    }
    return 0;
}
"""


def _inv_rows(T, axis, ang, s):
    a = np.asarray(axis, np.float64)
    R = np.eye(3)
    if ang != 0.0:
        a = a / np.linalg.norm(a)
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        R = np.cos(ang) * np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * np.outer(a, a)
    M = np.eye(4)
    M[:3, :3] = R * s
    M[:3, 3] = T
    return np.linalg.inv(M)[:3, :4].reshape(-1)


def test_boundary_object_animation(tmp_path):
    """Boundary-object transformations of the host scene reader: a static translated,
    scaled sphere and a box rotating about x by linear keyframes (0 -> 180 -> 360 degrees
    over frames 2..6, periodic from frame 2), checked against the same matrices built in
    numpy; a translation animated by a clamped cubic spline against scipy's."""
    import json
    from scipy.interpolate import CubicSpline
    scene = {"AdditionalBoundaryObjects": [
        {"GeometryType": "Sphere", "Translation": [0.5, 0.4, 0.5], "Scale": 0.7},
        {"GeometryType": "Box", "BoxMin": [-0.4, -0.2, -0.4], "BoxMax": [0.4, 0.2, 0.4],
         "Translation": [0.5, 0.5, 0.5],
         "Animation": {"Periodic": True, "StartFrame": 2, "CubicInterpolationRotation": False,
                       "KeyFrames": [{"Frame": 2, "Translation": [0.5, 0.5, 0.5], "RotationAxisAngle": [1, 0, 0, 0]},
                                     {"Frame": 4, "Translation": [0.5, 0.5, 0.5], "RotationAxisAngle": [1, 0, 0, 180]},
                                     {"Frame": 6, "Translation": [0.5, 0.5, 0.5], "RotationAxisAngle": [1, 0, 0, 360]}]}},
        {"GeometryType": "Sphere", "Scale": 0.6,
         "Animation": {"KeyFrames": [{"Frame": 1, "Translation": [0.4, 0.5, 0.5]},
                                     {"Frame": 3, "Translation": [0.6, 0.5, 0.5]},
                                     {"Frame": 5, "Translation": [0.5, 0.45, 0.5]}]}}]}
    (tmp_path / "s.json").write_text(json.dumps(scene))
    src = tmp_path / "a.cpp"
    src.write_text(ANIM_SELFTEST)
    exe = tmp_path / "a"
    host = bld.HOST
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(host), "-I", str(bld.INCLUDE), str(src),
                    str(host / "boundary_objects.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(tmp_path / "s.json")], capture_output=True, text=True, check=True).stdout
    rows = [l.split() for l in out.strip().splitlines()]
    assert rows[0][0] == "init" and len(rows) == 3 * 7
    got = {}
    for r in rows:
        got.setdefault(float(r[1]), []).append((int(r[2]), int(r[3]), np.array(r[4:16], float), float(r[16])))
    # static sphere: the same record at every time
    exp = _inv_rows([0.5, 0.4, 0.5], [0, 0, 1], 0.0, 0.7)
    for t, recs in got.items():
        assert recs[0][0] == 1 and recs[0][1] == 0
        np.testing.assert_allclose(recs[0][2], exp, atol=1e-6)
        assert abs(recs[0][3] - 0.7) < 1e-7
    # rotating box: linear angle in frames 2..6, periodic afterwards, static before frame 2
    def box_angle(t):
        f, frac = int(t), t - int(t)
        if f < 2:
            return None
        if f > 6:
            f = (f - 2) % 4 + 2
        return np.radians(90.0 * ((f + frac) - 2))
    for t, recs in got.items():
        tr, dyn, m, sc = recs[1]
        assert dyn == 1
        ang = box_angle(t) if t > 0 else None
        if ang is None:
            np.testing.assert_allclose(m, _inv_rows([0.5, 0.5, 0.5], [1, 0, 0], 0.0, 1.0), atol=1e-6)
        else:
            np.testing.assert_allclose(m, _inv_rows([0.5, 0.5, 0.5], [1, 0, 0], ang, 1.0), atol=2e-6)
    # cubic translation and scale: keyframe 0 (the object's own: origin, Scale 0.6) and
    # keyframes 1, 3, 5 (their Scale defaults to 1), zero end slopes
    xs = [0, 1, 3, 5]
    ys = np.array([[0, 0, 0], [0.4, 0.5, 0.5], [0.6, 0.5, 0.5], [0.5, 0.45, 0.5]])
    cs = CubicSpline(xs, ys, bc_type="clamped")
    css = CubicSpline(xs, [0.6, 1.0, 1.0, 1.0], bc_type="clamped")
    for t, recs in got.items():
        if t == 0 or t > 5:
            continue
        np.testing.assert_allclose(recs[2][2], _inv_rows(cs(t), [0, 0, 1], 0.0, float(css(t))), atol=2e-6)
        assert abs(recs[2][3] - float(css(t))) < 1e-6
