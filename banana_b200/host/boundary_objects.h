// Boundary objects of a scene ("AdditionalBoundaryObjects") and their keyframe animation,
// evaluated on the host into the world-to-object maps bnn_flip_set_boundaries takes.
//
//  * geometry: "Box" (BoxMin / BoxMax in object space) or "Sphere" (unit sphere scaled by
//    Scale), GeometryObjects.cpp:246-268,379-384;
//  * transformation translate * rotate(axis, angle) * scale of the current keyframe values
//    (Animation.h:199-231), RotationAxisAngle in degrees (GeometryObjects.cpp:155-158);
//  * "Animation": KeyFrames {Frame, Translation, RotationAxisAngle, Scale}, Periodic +
//    StartFrame, CubicInterpolation{Translation,Rotation,Scale} (GeometryObjects.cpp:163-195).
//    Keyframe 0 holds the object's own Translation / RotationAxisAngle / Scale; a keyframe
//    at frame 0 replaces it (Animation.h:73-80).  Each component is interpolated over the
//    keyframes by a cubic spline with zero end slopes, or piecewise linearly, and
//    continued past the ends by the end piece's polynomial (CubicSpline.h:240-380).
#pragma once

#include <string>
#include <vector>

#include <banana_b200.h>

namespace bnnhost {

struct Json;

// One-dimensional interpolant through (x[i], y[i]), x strictly increasing: piecewise
// cubic a h^3 + b h^2 + c h + y on [x[i], x[i+1]) with a continuous second derivative and
// y'(x0) = y'(xn) = 0, or piecewise linear; beyond the ends the end piece's quadratic /
// linear part continues.
class KeySpline {
public:
    void fit(const std::vector<double>& x, const std::vector<double>& y, bool cubic);
    double operator()(double t) const;

private:
    std::vector<double> m_x, m_y, m_a, m_b, m_c;
    double m_b0 = 0, m_c0 = 0;
};

struct KeyFrame {
    unsigned frame = 0;
    double translation[3] = {0, 0, 0};
    double rotation[4] = {0, 0, 1, 0};  // axis, angle in radians
    double scale = 1;
};

struct BoundaryObjectSpec {
    std::string name;
    int geometry = BNN_GEOMETRY_BOX;
    float boxMin[3] = {-1, -1, -1};
    float boxMax[3] = {1, 1, 1};
    bool transformed = false;  // an object-level Translation / Rotation / Scale was given
    bool dynamic = false;      // an "Animation" was given
    bool periodic = false;
    unsigned startFrame = 0, maxFrame = 0;
    std::vector<KeyFrame> keys{KeyFrame{}};
    KeySpline spline[8];        // translation x3, rotation axis x3 + angle, scale
    bnn_boundary_object current{};  // the C ABI record of the current transformation

    void makeReady(bool cubicT, bool cubicR, bool cubicS);
    // GeometryObject::updateTransformation(frame, fraction) (GeometryObjects.cpp:121-138);
    // false when nothing moves (frame > 0 with a single keyframe)
    bool update(unsigned frame, double fraction);
    // current <- the world-to-object map of translate(T) * rotate(R) * scale(s)
    void setRecord(const double T[3], const double R[4], double s, double uniformScale);
};

// ParticleSolver::generateBoundaries' parser (ParticleSolver.cpp:242-260) for Box / Sphere
// objects; other geometry types are refused with a message in `error`
std::vector<BoundaryObjectSpec> parse_boundary_objects(const Json& scene, std::string& error);

} // namespace bnnhost
