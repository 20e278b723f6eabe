// Anisotropic particle kernels for surface reconstruction: the reference's
// AnisotropicKernelGenerator<3, float>::computeAniKernels
// (Simulation/SurfaceReconstruction/AniKernelGenerator.cpp:53-101), which
// PIC_Solver::saveFrameData runs when "AniKernel" is among the saved data
// (Simulation/ParticleSolvers/PICFluid/PIC_Solver.cpp:248-252).
//
// Per particle p, over its neighbours q (|p - q|^2 < r^2, q != p; r = kernelRatio x
// particleRadius) and with W(d) = 1 - (|d| / r)^3:
//   weighted mean m = (p + sum W(p-q) q) / (1 + sum W(p-q)), centre = lerp(p, m, blend);
//   fewer than `threshold` neighbours: kernel = defaultSpraySize x identity;
//   else C = sum W(q-m) (q-m)(q-m)^T / (1 + sum W(q-m)), C = Q diag(S) Q^T with S sorted
//   descending, S[1,2] = max(S[1,2], S[0] / axisRatio), S *= cbrt(1 / prod S),
//   kernel = Q diag(S) Q^T (column-major, glm::mat3 memory order).
//
// One thread per particle in cell-sorted order.  Both passes walk the cell rows around the
// particle (z outer, y inner) and, in each row, the sorted particles of the cells its
// kernel sphere can reach, so every thread sums its neighbours in the canonical order
// (rows, then cell-sorted order).  Rows and cells that provably hold no neighbour are
// skipped; the margins cover the float rounding of the cell index (see row_range).  The
// accumulation is branch-free: a candidate outside the sphere adds a weight of 0, which
// leaves every sum unchanged (none of them can be -0), except the weighted mean, which is
// selected.  The covariance is symmetric positive semi-definite, so its SVD is its
// eigen-decomposition; a cyclic Jacobi iteration gives it, and the cube root is Newton's
// iteration in double precision, so the whole pass uses only correctly rounded
// operations and matches the CPU restatement bit for bit.
#include "bnn_internal.cuh"

#include <cfloat>
#include <cmath>
#include <cstring>

namespace bnn {

namespace {

struct AnisoArgs {
    float r2;         // kernel radius squared (float product, as the reference)
    float r2m;        // r2 (1 + 1e-4): the pruning radius squared
    float rinv;       // 1 / r
    float blend, axisRatio, spray;
    uint32_t threshold;
    int R;            // cell rows / columns a neighbour can lie away
    float margin;     // 0.01 cell: bound on how far a point's cell index can be off its position
};

__device__ __forceinline__ float kernel_w(float d2, float rinv) {
    const float t = sqrtf(d2) * rinv;
    return 1.0f - t * t * t;
}

// The sorted-index range [s, e) of cell row (j, k) that may hold neighbours of p.  A
// point stored in interior cell c lies within c * dx - margin .. (c + 1) * dx + margin
// of bmin (the truncated cell index is off by at most ~1e-4 cell for grids up to 1024
// cells); the border rows and columns also hold any point clamped onto them.  Rows whose
// distance from p exceeds the pruning radius hold no neighbour, and within a row only the
// cells within the chord (plus the margin) can.
__device__ __forceinline__ bool row_range(const AnisoGrid& g, const AnisoArgs& a, const uint32_t* __restrict__ cellStart,
                                          float px, float py, float pz, int j, int k, uint32_t& s, uint32_t& e) {
    if(j < 0 || j >= g.G[1] || k < 0 || k >= g.G[2]) return false;
    const float ylo = j == 0 ? -INFINITY : g.bmin[1] + (float)j * g.dx - a.margin;
    const float yhi = j == g.G[1] - 1 ? INFINITY : g.bmin[1] + (float)(j + 1) * g.dx + a.margin;
    const float zlo = k == 0 ? -INFINITY : g.bmin[2] + (float)k * g.dx - a.margin;
    const float zhi = k == g.G[2] - 1 ? INFINITY : g.bmin[2] + (float)(k + 1) * g.dx + a.margin;
    const float dy = fmaxf(0.0f, fmaxf(ylo - py, py - yhi));
    const float dz = fmaxf(0.0f, fmaxf(zlo - pz, pz - zhi));
    const float dyz = dy * dy + dz * dz;
    if(!(dyz < a.r2m)) return false;
    const float ext = sqrtf(a.r2m - dyz) + a.margin;
    int i0 = (int)floorf((px - ext - g.bmin[0]) / g.dx);
    int i1 = (int)floorf((px + ext - g.bmin[0]) / g.dx);
    i0 = i0 < 0 ? 0 : i0;
    i1 = i1 > g.G[0] - 1 ? g.G[0] - 1 : i1;
    if(i0 > i1) return false;
    const size_t row = ((size_t)k * g.G[1] + j) * g.G[0];
    s = cellStart[row + i0];
    e = cellStart[row + i1 + 1];
    return s < e;
}

// Newton's iteration for the cube root, x <- (2x + m / x^2) / 3, on the mantissa in
// [0.5, 4) with the exponent split off exactly; 0, inf and NaN map to themselves.
__device__ __forceinline__ double cbrt_newton(double y) {
    if(!(y == y) || y == 0.0 || isinf(y)) return y;
    const bool neg = y < 0.0;
    int e;
    double m = frexp(neg ? -y : y, &e);
    int q = e / 3, r = e % 3;
    if(r < 0) { r += 3; --q; }
    m = ldexp(m, r);
    double x = 1.0;
#pragma unroll 1
    for(int it = 0; it < 8; ++it) x = (2.0 * x + m / (x * x)) / 3.0;
    x = ldexp(x, q);
    return neg ? -x : x;
}

// One Jacobi rotation annihilating a[P][Q] (symmetric a, eigenvectors in v's columns)
template<int P, int Q>
__device__ __forceinline__ void jacobi_rotate(float a[3][3], float v[3][3]) {
    constexpr int R = 3 - P - Q;
    const float apq = a[P][Q];
    if(apq == 0.0f) return;
    const float app = a[P][P], aqq = a[Q][Q];
    if(fabsf(apq) < 1e-9f * (fabsf(app) + fabsf(aqq))) {
        a[P][Q] = a[Q][P] = 0.0f;
        return;
    }
    const float tau = (aqq - app) / (2.0f * apq);
    float t;
    if(fabsf(tau) > 1e15f) t = 0.5f / tau;
    else {
        t = 1.0f / (fabsf(tau) + sqrtf(1.0f + tau * tau));
        if(tau < 0.0f) t = -t;
    }
    const float c = 1.0f / sqrtf(1.0f + t * t);
    const float s = t * c;
    a[P][P] = app - t * apq;
    a[Q][Q] = aqq + t * apq;
    a[P][Q] = a[Q][P] = 0.0f;
    const float arp = a[R][P], arq = a[R][Q];
    a[R][P] = a[P][R] = c * arp - s * arq;
    a[R][Q] = a[Q][R] = s * arp + c * arq;
#pragma unroll
    for(int k = 0; k < 3; ++k) {
        const float vkp = v[k][P], vkq = v[k][Q];
        v[k][P] = c * vkp - s * vkq;
        v[k][Q] = s * vkp + c * vkq;
    }
}

template<int I, int J>
__device__ __forceinline__ void sort_pair(float lam[3], float v[3][3]) {
    if(lam[I] < lam[J]) {
        const float t = lam[I]; lam[I] = lam[J]; lam[J] = t;
#pragma unroll
        for(int k = 0; k < 3; ++k) { const float u = v[k][I]; v[k][I] = v[k][J]; v[k][J] = u; }
    }
}

// AniKernelGenerator.cpp:91-98 on the covariance a (destroyed); out column-major
__device__ __forceinline__ void kernel_matrix(float a[3][3], float axisRatio, float out[9]) {
    float v[3][3] = {{1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}};
#pragma unroll 1
    for(int sweep = 0; sweep < 10; ++sweep) {
        if(a[0][1] == 0.0f && a[0][2] == 0.0f && a[1][2] == 0.0f) break;
        jacobi_rotate<0, 1>(a, v);
        jacobi_rotate<0, 2>(a, v);
        jacobi_rotate<1, 2>(a, v);
    }
    float S[3] = {a[0][0], a[1][1], a[2][2]};
    sort_pair<0, 1>(S, v);
    sort_pair<1, 2>(S, v);
    sort_pair<0, 1>(S, v);
    const float lo = S[0] / axisRatio;
    S[1] = S[1] < lo ? lo : S[1];
    S[2] = S[2] < lo ? lo : S[2];
    const float prod = S[0] * S[1] * S[2];
    const float sc = (float)cbrt_newton((double)(1.0f / prod));
#pragma unroll
    for(int i = 0; i < 3; ++i) S[i] = S[i] * sc;
#pragma unroll
    for(int c = 0; c < 3; ++c)
#pragma unroll
        for(int r = 0; r < 3; ++r)
            out[c * 3 + r] = v[r][0] * S[0] * v[c][0] + v[r][1] * S[1] * v[c][1] + v[r][2] * S[2] * v[c][2];
}

__global__ void __launch_bounds__(128) k_aniso(int n, const float4* __restrict__ pos, const uint32_t* __restrict__ ids,
                                               const uint32_t* __restrict__ cellStart, AnisoGrid g, AnisoArgs a,
                                               float* __restrict__ outC, float* __restrict__ outM,
                                               unsigned* __restrict__ counters) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < n;
    const float4 P = active ? pos[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    int cj, ck;
    {
        int c[3] = {(int)((P.x - g.bmin[0]) / g.dx), (int)((P.y - g.bmin[1]) / g.dx), (int)((P.z - g.bmin[2]) / g.dx)};
        bool out = false;
#pragma unroll
        for(int d = 0; d < 3; ++d) {
            if(c[d] < 0) { c[d] = 0; out = true; }
            if(c[d] > g.G[d] - 1) { c[d] = g.G[d] - 1; out = true; }
        }
        // the pruning assumes every point lies in the grid it was sorted on
        if(active && out) atomicAdd(counters + 1, 1u);
        cj = c[1];
        ck = c[2];
    }
    const int R = a.R;
    const uint32_t self = (uint32_t)p;

    // pass 1: neighbour count and weighted mean (AniKernelGenerator.cpp:65-75)
    float sw = 1.0f, mx = P.x, my = P.y, mz = P.z;
    uint32_t cnt = 0;
    for(int dz = -R; dz <= R; ++dz)
        for(int dy = -R; dy <= R; ++dy) {
            uint32_t s = 0, e = 0;
            if(active) row_range(g, a, cellStart, P.x, P.y, P.z, cj + dy, ck + dz, s, e);
#pragma unroll 2
            for(uint32_t q = s; q < e; ++q) {
                const float4 Q = __ldg(pos + q);
                const float ex = P.x - Q.x, ey = P.y - Q.y, ez = P.z - Q.z;
                const float d2 = ex * ex + ey * ey + ez * ez;
                const bool hit = d2 < a.r2 && q != self;
                const float w = hit ? kernel_w(d2, a.rinv) : 0.0f;
                sw = sw + w;
                cnt += hit ? 1u : 0u;
                const float ax = mx + w * Q.x, ay = my + w * Q.y, az = mz + w * Q.z;
                mx = hit ? ax : mx;
                my = hit ? ay : my;
                mz = hit ? az : mz;
            }
        }
    const float wx = mx / sw, wy = my / sw, wz = mz / sw;
    const uint32_t id = active ? ids[p] : 0u;
    if(active) {
        // MathHelpers::lerp (MathHelpers.h:549-551)
        const float f = a.blend, omf = 1.0f - f;
        outC[3 * (size_t)id] = omf * P.x + f * wx;
        outC[3 * (size_t)id + 1] = omf * P.y + f * wy;
        outC[3 * (size_t)id + 2] = omf * P.z + f * wz;
    }
    const bool need = active && cnt >= a.threshold;
    const unsigned sprayMask = __ballot_sync(0xffffffffu, active && !need);
    if((threadIdx.x & 31) == 0 && sprayMask) atomicAdd(counters, (unsigned)__popc(sprayMask));
    if(active && !need) {
        float* M = outM + 9 * (size_t)id;
#pragma unroll
        for(int e = 0; e < 9; ++e) M[e] = (e % 4 == 0) ? a.spray : 0.0f;
    }
    if(!__any_sync(0xffffffffu, need)) return;

    // pass 2: covariance about the weighted mean (AniKernelGenerator.cpp:80-89)
    float sw2 = 1.0f, c00 = 0.f, c01 = 0.f, c02 = 0.f, c11 = 0.f, c12 = 0.f, c22 = 0.f;
    for(int dz = -R; dz <= R; ++dz)
        for(int dy = -R; dy <= R; ++dy) {
            uint32_t s = 0, e = 0;
            if(need) row_range(g, a, cellStart, P.x, P.y, P.z, cj + dy, ck + dz, s, e);
#pragma unroll 2
            for(uint32_t q = s; q < e; ++q) {
                const float4 Q = __ldg(pos + q);
                const float ex = P.x - Q.x, ey = P.y - Q.y, ez = P.z - Q.z;
                const float d2 = ex * ex + ey * ey + ez * ez;
                const float x0 = Q.x - wx, x1 = Q.y - wy, x2 = Q.z - wz;
                const float dm = x0 * x0 + x1 * x1 + x2 * x2;
                const bool hit = d2 < a.r2 && q != self && dm < a.r2;
                const float w = hit ? kernel_w(dm, a.rinv) : 0.0f;
                sw2 = sw2 + w;
                c00 = c00 + w * (x0 * x0);
                c01 = c01 + w * (x0 * x1);
                c02 = c02 + w * (x0 * x2);
                c11 = c11 + w * (x1 * x1);
                c12 = c12 + w * (x1 * x2);
                c22 = c22 + w * (x2 * x2);
            }
        }
    if(!need) return;
    float C[3][3];
    C[0][0] = c00 / sw2; C[0][1] = c01 / sw2; C[0][2] = c02 / sw2;
    C[1][1] = c11 / sw2; C[1][2] = c12 / sw2; C[2][2] = c22 / sw2;
    C[1][0] = C[0][1]; C[2][0] = C[0][2]; C[2][1] = C[1][2];
    float M[9];
    kernel_matrix(C, a.axisRatio, M);
    float* out = outM + 9 * (size_t)id;
#pragma unroll
    for(int e = 0; e < 9; ++e) out[e] = M[e];
}

__global__ void k_pack_sorted(const float* __restrict__ pos, const uint32_t* __restrict__ order, uint32_t n,
                              float4* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const uint32_t p = order[i];
    out[i] = make_float4(pos[3 * (size_t)p], pos[3 * (size_t)p + 1], pos[3 * (size_t)p + 2], 0.0f);
}

// order-preserving float <-> uint keys for atomic min / max
__device__ __forceinline__ unsigned fkey(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
float fkey_inv(unsigned k) {
    const unsigned b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// Bounding box of the points (keys[0..2] min, keys[3..5] max) and a count of non-finite
// coordinates (keys[6])
__global__ void __launch_bounds__(256) k_bounds(const float* __restrict__ pos, uint32_t n, unsigned* keys) {
    unsigned mn[3] = {~0u, ~0u, ~0u}, mx[3] = {0u, 0u, 0u}, bad = 0;
    for(size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
#pragma unroll
        for(int d = 0; d < 3; ++d) {
            const float v = pos[3 * p + d];
            if(!isfinite(v)) { ++bad; continue; }
            const unsigned k = fkey(v);
            mn[d] = min(mn[d], k);
            mx[d] = max(mx[d], k);
        }
#pragma unroll
    for(int d = 0; d < 3; ++d)
        for(int off = 16; off > 0; off >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], off));
            mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], off));
        }
    for(int off = 16; off > 0; off >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, off);
    if((threadIdx.x & 31) == 0) {
        for(int d = 0; d < 3; ++d) { atomicMin(keys + d, mn[d]); atomicMax(keys + 3 + d, mx[d]); }
        if(bad) atomicAdd(keys + 6, bad);
    }
}

AnisoArgs make_args(const bnn_aniso_params& prm, float dx) {
    AnisoArgs a;
    // AnisotropicKernelGenerator constructor (AniKernelGenerator.cpp:30-42)
    const float r = prm.kernel_ratio * prm.particle_radius;
    a.r2 = r * r;
    a.r2m = a.r2 * (1.0f + 1e-4f);
    a.rinv = 1.0f / r;
    a.blend = prm.position_blending;
    a.axisRatio = prm.axis_ratio;
    a.spray = prm.default_spray_size;
    a.threshold = prm.neighbor_threshold;
    a.R = (int)(r / dx) + 2;
    a.margin = 0.01f * dx;
    return a;
}

} // namespace

bnn_aniso_params aniso_defaults(float particleRadius) {
    // AniKernelGenerator.h:41-45 (constructor defaults) and :51 (setParameters defaults)
    bnn_aniso_params p;
    p.particle_radius = particleRadius;
    p.kernel_ratio = 8.0f;
    p.default_spray_size = 0.75f;
    p.position_blending = 0.5f;
    p.axis_ratio = 8.0f;
    p.neighbor_threshold = 25u;
    return p;
}

int aniso_check_params(const bnn_aniso_params& p) {
    const float r = p.kernel_ratio * p.particle_radius;
    if(!(r > 0.0f) || !std::isfinite(r) || !(p.axis_ratio > 0.0f)) return BNN_ERR_INVALID_ARGUMENT;
    return BNN_OK;
}

// The pass over cell-sorted points pos (float4 x, y, z, -), ids = input index of each
// sorted point, cellStart = C + 1 offsets of grid g.  counters[0] receives the spray
// points, counters[1] the points outside g (both must be zeroed by the caller).
void launch_aniso(int n, const float4* pos, const uint32_t* ids, const uint32_t* cellStart, const AnisoGrid& g,
                  const bnn_aniso_params& prm, float* outC, float* outM, unsigned* counters, cudaStream_t s) {
    if(n <= 0) return;
    const AnisoArgs a = make_args(prm, g.dx);
    { k_aniso<<<(n + 127) / 128, 128, 0, s>>>(n, pos, ids, cellStart, g, a, outC, outM, counters); bnn_note_launch(); }
}

} // namespace bnn

using namespace bnn;

namespace {
struct DevMem {
    void* p = nullptr;
    ~DevMem() { if(p) cudaFree(p); }
    cudaError_t alloc(size_t b) { return cudaMalloc(&p, b ? b : 1); }
    template<class T> T* as() { return (T*)p; }
};
} // namespace

extern "C" int bnn_aniso_default_params(float particle_radius, bnn_aniso_params* out) {
    if(!out) return BNN_ERR_INVALID_ARGUMENT;
    *out = aniso_defaults(particle_radius);
    return BNN_OK;
}

extern "C" int bnn_anisotropic_kernels(const float* pos_dev, uint32_t n, const bnn_aniso_params* params,
                                       float* centers_dev, float* matrices_dev, bnn_aniso_stats* stats, void* stream) {
    if(!params || (n && (!pos_dev || !centers_dev || !matrices_dev))) return BNN_ERR_INVALID_ARGUMENT;
    int rc = aniso_check_params(*params);
    if(rc != BNN_OK) return rc;
    if(stats) std::memset(stats, 0, sizeof(*stats));
    if(n == 0) return BNN_OK;
    cudaStream_t s = (cudaStream_t)stream;
    // bounding box of the points -> the cell grid (cells of a quarter kernel radius)
    DevMem keys;
    BNN_CUDA_CHECK(keys.alloc(8 * sizeof(unsigned)));
    const unsigned init[8] = {~0u, ~0u, ~0u, 0u, 0u, 0u, 0u, 0u};
    BNN_CUDA_CHECK(cudaMemcpyAsync(keys.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    { k_bounds<<<4 * 148, 256, 0, s>>>(pos_dev, n, keys.as<unsigned>()); bnn_note_launch(); }
    unsigned hk[8];
    BNN_CUDA_CHECK(cudaMemcpyAsync(hk, keys.p, sizeof(hk), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    if(hk[6]) {
        bnn_set_error("bnn_anisotropic_kernels: non-finite coordinates");
        return BNN_ERR_INVALID_ARGUMENT;
    }
    const float r = params->kernel_ratio * params->particle_radius;
    AnisoGrid g;
    float lo[3], hi[3];
    for(int d = 0; d < 3; ++d) { lo[d] = fkey_inv(hk[d]); hi[d] = fkey_inv(hk[3 + d]); g.bmin[d] = lo[d]; }
    float cell = 0.25f * r;
    for(;;) {
        size_t C = 1;
        for(int d = 0; d < 3; ++d) {
            const float t = (hi[d] - lo[d]) / cell;
            g.G[d] = (int)t + 1;
            C *= (size_t)g.G[d];
        }
        if(C <= ((size_t)1 << 27)) break;
        cell = cell * std::cbrt((float)C / (float)((size_t)1 << 27)) * 1.01f;
    }
    g.dx = cell;
    const size_t C = (size_t)g.G[0] * g.G[1] * g.G[2];
    DevMem cid, order, start, pos4, cnt;
    BNN_CUDA_CHECK(cid.alloc((size_t)n * 4));
    BNN_CUDA_CHECK(order.alloc((size_t)n * 4));
    BNN_CUDA_CHECK(start.alloc((C + 1) * 4));
    BNN_CUDA_CHECK(pos4.alloc((size_t)n * sizeof(float4)));
    BNN_CUDA_CHECK(cnt.alloc(2 * sizeof(unsigned)));
    uint32_t oor = 0;
    rc = bnn_cell_sort(pos_dev, n, g.bmin, g.dx, g.G, cid.as<uint32_t>(), order.as<uint32_t>(), start.as<uint32_t>(),
                       &oor, stream);
    if(rc != BNN_OK) return rc;
    { k_pack_sorted<<<(n + 255) / 256, 256, 0, s>>>(pos_dev, order.as<uint32_t>(), n, pos4.as<float4>()); bnn_note_launch(); }
    BNN_CUDA_CHECK(cudaMemsetAsync(cnt.p, 0, 2 * sizeof(unsigned), s));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    launch_aniso((int)n, pos4.as<float4>(), order.as<uint32_t>(), start.as<uint32_t>(), g, *params, centers_dev,
                 matrices_dev, cnt.as<unsigned>(), s);
    cudaEventRecord(e1, s);
    unsigned hc[2];
    BNN_CUDA_CHECK(cudaMemcpyAsync(hc, cnt.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BNN_CUDA_CHECK(cudaGetLastError());
    if(stats) {
        for(int d = 0; d < 3; ++d) { stats->grid_bmin[d] = g.bmin[d]; stats->grid_dims[d] = g.G[d]; }
        stats->grid_cell_size = g.dx;
        stats->sprays = hc[0];
        stats->ms = ms;
    }
    if(oor || hc[1]) {
        bnn_set_error("bnn_anisotropic_kernels: a point fell outside its cell grid");
        return BNN_ERR_DEVICE_CHECK;
    }
    return BNN_OK;
}
