// =====================================================================================
//  TEST INFRASTRUCTURE ONLY -- the oracle for the anisotropic-kernel pass.
//
//  A CPU restatement of the reference's AnisotropicKernelGenerator<3, float>
//  (Simulation/SurfaceReconstruction/AniKernelGenerator.{h,cpp}; called from
//  PIC_Solver::saveFrameData, Simulation/ParticleSolvers/PICFluid/PIC_Solver.cpp:248-252)
//  in a fixed evaluation order, so the CUDA pass can be checked against it bit for bit.
//  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
//
//  What is the reference's and what is fixed here:
//   * weights, neighbour set, weighted mean, blended centre, spray threshold, covariance
//     and the kernel matrix U diag(S) V^T with S clamped to S[0] / axisRatio and scaled to
//     det 1 follow AniKernelGenerator.cpp:53-101 and .h:56-58 operation for operation;
//   * the neighbour sums run in a canonical order: the points are stably sorted by the
//     linear index of a uniform cell grid, and each point visits the cell rows around it
//     (z outer, y inner) and each row's points in sorted order.  The reference's order
//     comes from its CompactNSearch hash and thread schedule, so it has no single answer;
//   * the 3x3 SVD (ImplicitQRSVD, BananaCore/Banana/LinearAlgebra/ImplicitQRSVD.h:44-48)
//     is replaced by a cyclic Jacobi eigen-decomposition: the covariance is symmetric
//     positive semi-definite, so its SVD is its eigen-decomposition and
//     U diag(f(S)) V^T = Q diag(f(lambda)) Q^T does not depend on how it is factored;
//   * std::cbrt is replaced by Newton's iteration for the cube root in double precision
//     (exact IEEE operations only), rounded to float once.
//  tests/test_aniso_cpu.py checks this restatement against a direct numpy transcription of
//  the reference formulas (brute-force neighbour lists, LAPACK SVD in double precision).
//
//  Compile with -ffp-contract=off: every float operation is a single IEEE-rounded one.
// =====================================================================================
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc_aniso {

struct Params {
    float r2;         // kernel radius squared, (kernelRatio * particleRadius)^2 in float
    float rinv;       // 1 / kernel radius in float
    float blend;      // positionBlending
    float axisRatio;  // axisRatio
    float spray;      // defaultSpraySize
    uint32_t threshold;
};

// W2 (AniKernelGenerator.h:56): 1 - (sqrt(d2) / r)^3 inside the kernel radius
static inline float w2(float d2, const Params& P) {
    if(!(d2 < P.r2)) return 0.0f;
    const float t = std::sqrt(d2) * P.rinv;
    return 1.0f - t * t * t;
}

static inline float len2(float x, float y, float z) { return x * x + y * y + z * z; }

// Cube root by Newton's iteration x <- (2x + m / x^2) / 3 on the mantissa, with the
// exponent split off exactly (frexp / ldexp); inf, 0 and NaN map to themselves.
double cbrt_newton(double y) {
    if(!(y == y) || y == 0.0 || std::isinf(y)) return y;
    const bool neg = y < 0.0;
    int e;
    double m = std::frexp(neg ? -y : y, &e);  // m in [0.5, 1)
    int q = e / 3, r = e % 3;
    if(r < 0) { r += 3; --q; }
    m = std::ldexp(m, r);                     // m in [0.5, 4)
    double x = 1.0;
    for(int it = 0; it < 8; ++it) x = (2.0 * x + m / (x * x)) / 3.0;
    x = std::ldexp(x, q);
    return neg ? -x : x;
}

// One Jacobi rotation annihilating a[p][q] of the symmetric matrix a; v accumulates the
// rotations (columns = eigenvectors).
static void jacobi_rotate(float a[3][3], float v[3][3], int p, int q) {
    const float apq = a[p][q];
    if(apq == 0.0f) return;
    const float app = a[p][p], aqq = a[q][q];
    if(std::fabs(apq) < 1e-9f * (std::fabs(app) + std::fabs(aqq))) {
        a[p][q] = a[q][p] = 0.0f;
        return;
    }
    const float tau = (aqq - app) / (2.0f * apq);
    float t;
    if(std::fabs(tau) > 1e15f) t = 0.5f / tau;
    else {
        t = 1.0f / (std::fabs(tau) + std::sqrt(1.0f + tau * tau));
        if(tau < 0.0f) t = -t;
    }
    const float c = 1.0f / std::sqrt(1.0f + t * t);
    const float s = t * c;
    a[p][p] = app - t * apq;
    a[q][q] = aqq + t * apq;
    a[p][q] = a[q][p] = 0.0f;
    const int r = 3 - p - q;
    const float arp = a[r][p], arq = a[r][q];
    a[r][p] = a[p][r] = c * arp - s * arq;
    a[r][q] = a[q][r] = s * arp + c * arq;
    for(int k = 0; k < 3; ++k) {
        const float vkp = v[k][p], vkq = v[k][q];
        v[k][p] = c * vkp - s * vkq;
        v[k][q] = s * vkp + c * vkq;
    }
}

// Eigenvalues (descending) and eigenvectors (columns of v) of a symmetric 3x3 matrix
void eig_sym3(float a[3][3], float v[3][3], float lam[3]) {
    for(int i = 0; i < 3; ++i)
        for(int j = 0; j < 3; ++j) v[i][j] = i == j ? 1.0f : 0.0f;
    for(int sweep = 0; sweep < 10; ++sweep) {
        if(a[0][1] == 0.0f && a[0][2] == 0.0f && a[1][2] == 0.0f) break;
        jacobi_rotate(a, v, 0, 1);
        jacobi_rotate(a, v, 0, 2);
        jacobi_rotate(a, v, 1, 2);
    }
    for(int i = 0; i < 3; ++i) lam[i] = a[i][i];
    auto swp = [&](int i, int j) {
        if(lam[i] < lam[j]) {
            float t = lam[i]; lam[i] = lam[j]; lam[j] = t;
            for(int k = 0; k < 3; ++k) { float u = v[k][i]; v[k][i] = v[k][j]; v[k][j] = u; }
        }
    };
    swp(0, 1); swp(1, 2); swp(0, 1);
}

// Kernel matrix from the covariance (AniKernelGenerator.cpp:91-98); out is column-major
// (glm::mat3 memory order: out[c * 3 + r] = M[row r][column c])
void kernel_matrix(float C[3][3], float axisRatio, float* out) {
    float v[3][3], S[3];
    eig_sym3(C, v, S);
    const float lo = S[0] / axisRatio;
    for(int i = 1; i < 3; ++i) S[i] = S[i] < lo ? lo : S[i];  // std::max(S[i], lo)
    const float prod = S[0] * S[1] * S[2];
    const float sc = (float)cbrt_newton((double)(1.0f / prod));
    for(int i = 0; i < 3; ++i) S[i] = S[i] * sc;
    for(int c = 0; c < 3; ++c)
        for(int r = 0; r < 3; ++r)
            out[c * 3 + r] = v[r][0] * S[0] * v[c][0] + v[r][1] * S[1] * v[c][1] + v[r][2] * S[2] * v[c][2];
}

} // namespace orc_aniso

using namespace orc_aniso;

extern "C" {

// AnisotropicKernelGenerator::computeAniKernels over pos (n x 3, AoS) on the cell grid
// (bmin, cellSize, ncells; Grid::getCellIdx truncation, clamped onto the border).  Writes
// centres (n x 3) and kernel matrices (n x 9, column-major) in input order; returns the
// number of points below the neighbour threshold (the spray points).
uint32_t orc_aniso_kernels(const float* pos, uint32_t n, const float* bmin, float cellSize, const int32_t* ncells,
                           float particleRadius, float kernelRatio, float spray, float blend, float axisRatio,
                           uint32_t threshold, float* centers, float* mats) {
    // AnisotropicKernelGenerator constructor (AniKernelGenerator.cpp:30-42)
    const float r = kernelRatio * particleRadius;
    Params P{r * r, 1.0f / r, blend, axisRatio, spray, threshold};
    const int G[3] = {ncells[0], ncells[1], ncells[2]};
    const size_t C = (size_t)G[0] * G[1] * G[2];
    // stable cell sort: by linear cell, ties in input order
    std::vector<uint32_t> cell(n), start(C + 1, 0), order(n);
    std::vector<int> cc(3 * (size_t)n);
    for(uint32_t p = 0; p < n; ++p) {
        int c[3];
        for(int d = 0; d < 3; ++d) {
            c[d] = (int)((pos[3 * (size_t)p + d] - bmin[d]) / cellSize);
            c[d] = c[d] < 0 ? 0 : (c[d] > G[d] - 1 ? G[d] - 1 : c[d]);
            cc[3 * (size_t)p + d] = c[d];
        }
        cell[p] = (uint32_t)(((size_t)c[2] * G[1] + c[1]) * G[0] + c[0]);
        start[cell[p] + 1]++;
    }
    for(size_t c = 0; c < C; ++c) start[c + 1] += start[c];
    {
        std::vector<uint32_t> fill(start.begin(), start.end() - 1);
        for(uint32_t p = 0; p < n; ++p) order[fill[cell[p]]++] = p;
    }
    std::vector<float> sp(3 * (size_t)n);
    std::vector<uint32_t> slotOf(n);
    for(uint32_t s = 0; s < n; ++s) {
        slotOf[order[s]] = s;
        for(int d = 0; d < 3; ++d) sp[3 * (size_t)s + d] = pos[3 * (size_t)order[s] + d];
    }
    // every point within the kernel radius lies within R cells along each axis
    const int R = (int)(r / cellSize) + 2;
    uint32_t sprays = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : sprays)
    for(int64_t ip = 0; ip < (int64_t)n; ++ip) {
        const uint32_t p = (uint32_t)ip;
        const uint32_t self = slotOf[p];
        const float px = pos[3 * (size_t)p], py = pos[3 * (size_t)p + 1], pz = pos[3 * (size_t)p + 2];
        const int ci = cc[3 * (size_t)p], cj = cc[3 * (size_t)p + 1], ck = cc[3 * (size_t)p + 2];
        // visits the neighbours (|p - q|^2 < r^2, q != p) in canonical order
        auto walk = [&](auto&& f) {
            for(int dz = -R; dz <= R; ++dz) {
                const int k = ck + dz;
                if(k < 0 || k >= G[2]) continue;
                for(int dy = -R; dy <= R; ++dy) {
                    const int j = cj + dy;
                    if(j < 0 || j >= G[1]) continue;
                    const int i0 = ci - R < 0 ? 0 : ci - R, i1 = ci + R > G[0] - 1 ? G[0] - 1 : ci + R;
                    const size_t row = ((size_t)k * G[1] + j) * G[0];
                    for(uint32_t s = start[row + i0]; s < start[row + i1 + 1]; ++s) {
                        if(s == self) continue;
                        const float qx = sp[3 * (size_t)s], qy = sp[3 * (size_t)s + 1], qz = sp[3 * (size_t)s + 2];
                        if(len2(px - qx, py - qy, pz - qz) < P.r2) f(qx, qy, qz);
                    }
                }
            }
        };
        // weighted mean of positions (AniKernelGenerator.cpp:65-75)
        float sumW = 1.0f, wx = px, wy = py, wz = pz;
        uint32_t nn = 0;
        walk([&](float qx, float qy, float qz) {
            const float w = w2(len2(px - qx, py - qy, pz - qz), P);
            sumW = sumW + w;
            wx = wx + w * qx; wy = wy + w * qy; wz = wz + w * qz;
            ++nn;
        });
        wx = wx / sumW; wy = wy / sumW; wz = wz / sumW;
        // MathHelpers::lerp (MathHelpers.h:549-551)
        const float f = P.blend;
        centers[3 * (size_t)p] = (1.0f - f) * px + f * wx;
        centers[3 * (size_t)p + 1] = (1.0f - f) * py + f * wy;
        centers[3 * (size_t)p + 2] = (1.0f - f) * pz + f * wz;
        float* M = mats + 9 * (size_t)p;
        if(nn < P.threshold) {
            // MatNxN(defaultSpraySize): a scaled identity
            for(int e = 0; e < 9; ++e) M[e] = (e % 4 == 0) ? P.spray : 0.0f;
            ++sprays;
            continue;
        }
        // covariance about the weighted mean (AniKernelGenerator.cpp:80-89)
        float sw = 1.0f;
        float Cm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        walk([&](float qx, float qy, float qz) {
            const float x[3] = {qx - wx, qy - wy, qz - wz};
            const float w = w2(len2(x[0], x[1], x[2]), P);
            sw = sw + w;
            for(int c = 0; c < 3; ++c)
                for(int rr = 0; rr < 3; ++rr) Cm[rr][c] = Cm[rr][c] + w * (x[rr] * x[c]);
        });
        for(int c = 0; c < 3; ++c)
            for(int rr = 0; rr < 3; ++rr) Cm[rr][c] = Cm[rr][c] / sw;
        kernel_matrix(Cm, P.axisRatio, M);
    }
    return sprays;
}

// The pieces on their own, for the unit checks
double orc_cbrt_newton(double y) { return cbrt_newton(y); }
void orc_aniso_kernel_matrix(const float* cov9, float axisRatio, float* out9) {
    float C[3][3];
    for(int c = 0; c < 3; ++c)
        for(int r = 0; r < 3; ++r) C[r][c] = cov9[c * 3 + r];
    kernel_matrix(C, axisRatio, out9);
}

} // extern "C"
