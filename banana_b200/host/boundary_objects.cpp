// Boundary objects and their keyframe animation: see boundary_objects.h.
#include "boundary_objects.h"

#include "json_lite.h"

#include <algorithm>
#include <cmath>

namespace bnnhost {

// Cubic pieces with a continuous second derivative: on [x_i, x_i+1), h = t - x_i,
// f = a_i h^3 + b_i h^2 + c_i h + y_i.  Matching values, slopes and curvatures at the
// inner knots gives, for the b_i,
//   h_{i-1}/3 b_{i-1} + 2 (h_{i-1} + h_i)/3 b_i + h_i/3 b_{i+1} = s_i - s_{i-1}
// (s_i the chord slopes), and a zero end slope gives (2 b_0 + b_1) h_0 = 3 s_0 and
// (b_{n-2} + 2 b_{n-1}) h_{n-2} = -3 s_{n-2}.  The tridiagonal system is solved by
// forward elimination and back substitution.
void KeySpline::fit(const std::vector<double>& x, const std::vector<double>& y, bool cubic) {
    m_x = x;
    m_y = y;
    const size_t n = x.size();
    m_a.assign(n, 0.0);
    m_b.assign(n, 0.0);
    m_c.assign(n, 0.0);
    if(n < 2) return;
    std::vector<double> h(n - 1), s(n - 1);
    for(size_t i = 0; i + 1 < n; ++i) {
        h[i] = x[i + 1] - x[i];
        s[i] = (y[i + 1] - y[i]) / h[i];
    }
    if(cubic) {
        std::vector<double> lo(n, 0.0), di(n, 0.0), up(n, 0.0), r(n, 0.0);
        di[0] = 2.0 * h[0];
        up[0] = h[0];
        r[0] = 3.0 * s[0];
        for(size_t i = 1; i + 1 < n; ++i) {
            lo[i] = h[i - 1] / 3.0;
            di[i] = 2.0 * (h[i - 1] + h[i]) / 3.0;
            up[i] = h[i] / 3.0;
            r[i] = s[i] - s[i - 1];
        }
        lo[n - 1] = h[n - 2];
        di[n - 1] = 2.0 * h[n - 2];
        r[n - 1] = -3.0 * s[n - 2];
        for(size_t i = 1; i < n; ++i) {
            const double m = lo[i] / di[i - 1];
            di[i] -= m * up[i - 1];
            r[i] -= m * r[i - 1];
        }
        m_b[n - 1] = r[n - 1] / di[n - 1];
        for(size_t i = n - 1; i-- > 0;) m_b[i] = (r[i] - up[i] * m_b[i + 1]) / di[i];
        for(size_t i = 0; i + 1 < n; ++i) {
            m_a[i] = (m_b[i + 1] - m_b[i]) / (3.0 * h[i]);
            m_c[i] = s[i] - (2.0 * m_b[i] + m_b[i + 1]) * h[i] / 3.0;
        }
    } else {
        for(size_t i = 0; i + 1 < n; ++i) m_c[i] = s[i];
    }
    // past the ends: the first piece's quadratic part on the left, the last piece's slope
    // and curvature at x_{n-1} on the right
    m_b0 = m_b[0];
    m_c0 = m_c[0];
    const double hl = h[n - 2];
    m_a[n - 1] = 0.0;
    m_c[n - 1] = 3.0 * m_a[n - 2] * hl * hl + 2.0 * m_b[n - 2] * hl + m_c[n - 2];
    if(!cubic) m_b[n - 1] = 0.0;
}

double KeySpline::operator()(double t) const {
    const size_t n = m_x.size();
    if(n == 0) return 0.0;
    if(n == 1) return m_y[0];
    const auto it = std::lower_bound(m_x.begin(), m_x.end(), t);
    const size_t idx = it == m_x.begin() ? 0 : (size_t)(it - m_x.begin()) - 1;
    const double h = t - m_x[idx];
    if(t < m_x[0]) return (m_b0 * h + m_c0) * h + m_y[0];
    if(t > m_x[n - 1]) return (m_b[n - 1] * h + m_c[n - 1]) * h + m_y[n - 1];
    return ((m_a[idx] * h + m_b[idx]) * h + m_c[idx]) * h + m_y[idx];
}

void BoundaryObjectSpec::makeReady(bool cubicT, bool cubicR, bool cubicS) {
    std::vector<double> xs, v[8];
    maxFrame = 0;
    for(const auto& k : keys) {
        if(periodic && k.frame < startFrame) continue;
        maxFrame = std::max(maxFrame, k.frame);
        xs.push_back((double)k.frame);
        for(int d = 0; d < 3; ++d) v[d].push_back(k.translation[d]);
        for(int d = 0; d < 4; ++d) v[3 + d].push_back(k.rotation[d]);
        v[7].push_back(k.scale);
    }
    for(int q = 0; q < 3; ++q) spline[q].fit(xs, v[q], cubicT);
    for(int q = 3; q < 7; ++q) spline[q].fit(xs, v[q], cubicR);
    spline[7].fit(xs, v[7], cubicS);
}

// world -> object map of translate(T) * rotate(R) * scale(s): (1/s) R^T (p - T)
void BoundaryObjectSpec::setRecord(const double T[3], const double R[4], double s, double uniformScale) {
    double a[3] = {R[0], R[1], R[2]};
    const double len = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double Rm[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if(len > 0.0 && R[3] != 0.0) {
        for(double& c : a) c /= len;
        const double c = std::cos(R[3]), sn = std::sin(R[3]), t = 1.0 - c;
        // Rodrigues' formula: c I + (1 - c) a a^T + sin [a]x
        Rm[0][0] = c + t * a[0] * a[0];
        Rm[0][1] = t * a[0] * a[1] - sn * a[2];
        Rm[0][2] = t * a[0] * a[2] + sn * a[1];
        Rm[1][0] = t * a[1] * a[0] + sn * a[2];
        Rm[1][1] = c + t * a[1] * a[1];
        Rm[1][2] = t * a[1] * a[2] - sn * a[0];
        Rm[2][0] = t * a[2] * a[0] - sn * a[1];
        Rm[2][1] = t * a[2] * a[1] + sn * a[0];
        Rm[2][2] = c + t * a[2] * a[2];
    }
    for(int r = 0; r < 3; ++r) {
        double off = 0.0;
        for(int c = 0; c < 3; ++c) {
            current.inv_transform[4 * r + c] = (float)(Rm[c][r] / s);
            off -= Rm[c][r] * T[c];
        }
        current.inv_transform[4 * r + 3] = (float)(off / s);
    }
    current.uniform_scale = (float)uniformScale;
    current.transformed = 1;
}

bool BoundaryObjectSpec::update(unsigned frame, double fraction) {
    if(frame > 0 && keys.size() == 1) return false;
    double T[3], R[4], s;
    if(keys.size() == 1 || (periodic && frame < startFrame)) {
        for(int d = 0; d < 3; ++d) T[d] = keys[0].translation[d];
        for(int d = 0; d < 4; ++d) R[d] = keys[0].rotation[d];
        s = keys[0].scale;
    } else {
        unsigned f = frame;
        if(periodic && f > maxFrame && maxFrame > startFrame) f = ((f - startFrame) % (maxFrame - startFrame)) + startFrame;
        const double x = (double)f + fraction;
        for(int d = 0; d < 3; ++d) T[d] = spline[d](x);
        for(int d = 0; d < 4; ++d) R[d] = spline[3 + d](x);
        s = spline[7](x);
    }
    // Animation::getUniformScale (Animation.h:240-252) wraps periodic frames by the last
    // keyframe alone
    double us = keys[0].scale;
    if(keys.size() > 1) {
        unsigned f = frame;
        if(periodic && f > maxFrame && maxFrame > 0) f = f % maxFrame;
        us = spline[7]((double)f + fraction);
    }
    setRecord(T, R, s, us);
    return true;
}

static bool num(const Json& j, const char* k, double& out) {
    if(!j.has(k) || j[k].kind != Json::Number) return false;
    out = j[k].num;
    return true;
}
static bool vec(const Json& j, const char* k, double* out, size_t n) {
    if(!j.has(k) || j[k].kind != Json::Array || j[k].size() < n) return false;
    for(size_t i = 0; i < n; ++i) out[i] = j[k][i].num;
    return true;
}
static bool flag(const Json& j, const char* k, bool& out) {
    if(!j.has(k) || j[k].kind != Json::Bool) return false;
    out = j[k].b;
    return true;
}

std::vector<BoundaryObjectSpec> parse_boundary_objects(const Json& scene, std::string& error) {
    std::vector<BoundaryObjectSpec> out;
    const Json& list = scene["AdditionalBoundaryObjects"];
    const double kDeg = 3.14159265358979323846 / 180.0;
    for(size_t i = 0; i < list.size(); ++i) {
        const Json& o = list[i];
        BoundaryObjectSpec b;
        const std::string type = o["GeometryType"].str;
        if(type == "Box" || type == "box" || type == "BOX") b.geometry = BNN_GEOMETRY_BOX;
        else if(type == "Sphere" || type == "sphere" || type == "SPHERE") b.geometry = BNN_GEOMETRY_SPHERE;
        else {
            error = "boundary object geometry '" + type + "' is not supported (Box and Sphere are)";
            return {};
        }
        b.name = o["UniqueName"].str;
        double v[4];
        if(vec(o, "BoxMin", v, 3)) for(int d = 0; d < 3; ++d) b.boxMin[d] = (float)v[d];
        if(vec(o, "BoxMax", v, 3)) for(int d = 0; d < 3; ++d) b.boxMax[d] = (float)v[d];
        KeyFrame& k0 = b.keys[0];
        if(vec(o, "Translation", v, 3)) {
            for(int d = 0; d < 3; ++d) k0.translation[d] = v[d];
            b.transformed = true;
        }
        if(vec(o, "RotationAxisAngle", v, 4) && v[3] != 0.0) {
            for(int d = 0; d < 3; ++d) k0.rotation[d] = v[d];
            k0.rotation[3] = v[3] * kDeg;
            b.transformed = true;
        }
        if(num(o, "Scale", v[0])) {
            k0.scale = v[0];
            b.transformed = true;
        }
        bool cubicT = true, cubicR = true, cubicS = true;
        if(o.has("Animation")) {
            const Json& a = o["Animation"];
            b.dynamic = true;
            flag(a, "CubicInterpolationTranslation", cubicT);
            flag(a, "CubicInterpolationRotation", cubicR);
            flag(a, "CubicInterpolationScale", cubicS);
            if(flag(a, "Periodic", b.periodic)) {
                double sf = 0;
                if(num(a, "StartFrame", sf)) b.startFrame = (unsigned)sf;
            }
            const Json& keys = a["KeyFrames"];
            for(size_t q = 0; q < keys.size(); ++q) {
                const Json& kj = keys[q];
                KeyFrame k;
                double fr = 0;
                num(kj, "Frame", fr);
                k.frame = (unsigned)fr;
                if(vec(kj, "Translation", v, 3)) for(int d = 0; d < 3; ++d) k.translation[d] = v[d];
                // every component of a keyframe's axis-angle goes through glm::radians
                if(vec(kj, "RotationAxisAngle", v, 4)) for(int d = 0; d < 4; ++d) k.rotation[d] = v[d] * kDeg;
                num(kj, "Scale", k.scale);
                if(k.frame == 0) b.keys[0] = k;
                else b.keys.push_back(k);
            }
            b.makeReady(cubicT, cubicR, cubicS);
        }
        b.current.geometry = b.geometry;
        b.current.dynamic = b.dynamic ? 1 : 0;
        for(int d = 0; d < 3; ++d) {
            b.current.box_min[d] = b.boxMin[d];
            b.current.box_max[d] = b.boxMax[d];
        }
        for(int q = 0; q < 12; ++q) b.current.inv_transform[q] = (q % 5 == 0) ? 1.0f : 0.0f;
        b.current.uniform_scale = 1.0f;
        b.current.transformed = 0;
        if(b.transformed) {
            // the static transformation the object is built with (keyframe 0)
            const KeyFrame& k = b.keys[0];
            b.setRecord(k.translation, k.rotation, k.scale, k.scale);
        }
        out.push_back(b);
    }
    return out;
}

} // namespace bnnhost
