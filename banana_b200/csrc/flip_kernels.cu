// Kernels of one FLIP / APIC / AFLIP sub-step on a single B200.
//
// Layout in HBM (one solver):
//   particles  SoA float x[], y[], z[], vx[], vy[], vz[] + uint32 id[] (original index),
//              kept physically sorted by cell (stable counting sort every step), plus the
//              grid coordinates gx[], gy[], gz[] of the sorted particles;
//   faces      u (G+1)GG, v G(G+1)G, w GG(G+1) floats in the reference's (k*Sy+j)*Sx+i
//              order, with uint8 valid flags and a ping-pong buffer for extrapolation;
//   cells      fluid SDF (float), cell histogram / start offsets (uint32), active index;
//   rows       the pressure system compacted to fluid cells (see pcg.cu).
//
// Every kernel is a gather: each output element is produced by exactly one thread, in
// the order the reference's serial loop would produce it, so no float atomics are used
// and results are bit-reproducible.
#include "bnn_internal.cuh"

namespace bnn {

// ----------------------------------------------------------------------------------
// Staggered-grid sampling
// ----------------------------------------------------------------------------------
// ArrayHelpers::interpolateValueLinear 3D (ArrayHelpers.cpp:91-102) with trilerp
// (MathHelpers.h:564-573)
__device__ __forceinline__ float interp_face(const float* __restrict__ a, int sx, int sy, int sz, float px, float py,
                                             float pz) {
    int i, j, k;
    float fi, fj, fk;
    bary(px, i, fi, sx);
    bary(py, j, fj, sy);
    bary(pz, k, fk, sz);
    // a face array holds fewer than 2^32 entries (cells < 2^31, at least 3 along x): the tap
    // index in 32 bits, then one pointer per stencil row
    const unsigned usx = (unsigned)sx, sxy = usx * (unsigned)sy;
    const float* r00 = a + ((unsigned)k * sxy + (unsigned)j * usx + (unsigned)i);
    const float* r10 = r00 + usx;
    const float* r01 = r00 + sxy;
    const float* r11 = r01 + usx;
    float v000 = __ldg(r00), v100 = __ldg(r00 + 1), v010 = __ldg(r10), v110 = __ldg(r10 + 1);
    float v001 = __ldg(r01), v101 = __ldg(r01 + 1), v011 = __ldg(r11), v111 = __ldg(r11 + 1);
    return lerpf(lerpf(lerpf(v000, v100, fi), lerpf(v010, v110, fi), fj),
                 lerpf(lerpf(v001, v101, fi), lerpf(v011, v111, fi), fj), fk);
}

// interp_face of a (*val) and the same trilinear sample of (a - o) (*diff), from one load of
// each tap: the grid velocity and the FLIP velocity change dVels = velocities - oldVels
// (FLIP_Solver.cpp:115-121), the difference formed tap by tap as if that array existed
__device__ __forceinline__ void interp_face_pair(const float* __restrict__ a, const float* __restrict__ o, int sx,
                                                 int sy, int sz, float px, float py, float pz, float* val, float* diff) {
    int i, j, k;
    float fi, fj, fk;
    bary(px, i, fi, sx);
    bary(py, j, fj, sy);
    bary(pz, k, fk, sz);
    // 32-bit tap index, then one pointer per stencil row (as interp_face)
    const unsigned usx = (unsigned)sx, sxy = usx * (unsigned)sy;
    const unsigned b = (unsigned)k * sxy + (unsigned)j * usx + (unsigned)i;
    const unsigned rows[4] = {0u, usx, sxy, sxy + usx};
    float va[8], vd[8];
#pragma unroll
    for(int r = 0; r < 4; ++r) {
        const float* pa = a + (b + rows[r]);
        const float* po = o + (b + rows[r]);
        va[2 * r] = __ldg(pa);
        vd[2 * r] = va[2 * r] - __ldg(po);
        va[2 * r + 1] = __ldg(pa + 1);
        vd[2 * r + 1] = va[2 * r + 1] - __ldg(po + 1);
    }
    *val = lerpf(lerpf(lerpf(va[0], va[1], fi), lerpf(va[2], va[3], fi), fj),
                 lerpf(lerpf(va[4], va[5], fi), lerpf(va[6], va[7], fi), fj), fk);
    *diff = lerpf(lerpf(lerpf(vd[0], vd[1], fi), lerpf(vd[2], vd[3], fi), fj),
                  lerpf(lerpf(vd[4], vd[5], fi), lerpf(vd[6], vd[7], fi), fj), fk);
}

// PIC_Solver::getVelocityFromGrid(gridPos) (PIC_Solver.cpp:1119-1133)
__device__ __forceinline__ void vel_from_grid(const GridDesc& g, const float* u, const float* v, const float* w,
                                              float gx, float gy, float gz, float out[3]) {
    out[0] = interp_face(u, g.G[0] + 1, g.G[1], g.G[2], gx, gy - 0.5f, gz - 0.5f);
    out[1] = interp_face(v, g.G[0], g.G[1] + 1, g.G[2], gx - 0.5f, gy, gz - 0.5f);
    out[2] = interp_face(w, g.G[0], g.G[1], g.G[2] + 1, gx - 0.5f, gy - 0.5f, gz);
}

// ----------------------------------------------------------------------------------
// Domain-box boundary (negative outside the box)
// ----------------------------------------------------------------------------------
// BoxObject::signedDistance with bNegativeInside = false (GeometryObjects.cpp:246-268)
__device__ __forceinline__ float box_sdf(const GridDesc& g, float x, float y, float z) {
    const float p[3] = {x, y, z};
    bool inside = true;
#pragma unroll
    for(int d = 0; d < 3; ++d)
        if(p[d] < g.boxMin[d] || p[d] > g.boxMax[d]) inside = false;
    float mind = FLT_MAX;
    if(inside) {
#pragma unroll
        for(int d = 0; d < 3; ++d) mind = smin(mind, smin(p[d] - g.boxMin[d], g.boxMax[d] - p[d]));
        mind = -mind;
    } else {
        float c[3];
#pragma unroll
        for(int d = 0; d < 3; ++d) c[d] = smax(smin(p[d], g.boxMax[d]), g.boxMin[d]);
        mind = sqrtf(length2f(p[0] - c[0], p[1] - c[1], p[2] - c[2]));
    }
    mind = -mind;
    return 1.0f * mind;
}

// BoundaryObject::constrainToBoundary (BoundaryObject.cpp:72-90) with the 8-point
// finite-difference gradient of GeometryObject::gradSignedDistance (GeometryObjects.cpp:37-85)
__device__ __forceinline__ void constrain_to_box(const GridDesc& g, float& x, float& y, float& z) {
    const float phiVal = box_sdf(g, x, y, z);
    if(phiVal < 0.f) {
        const float e = 1e-4f;
        float v000 = box_sdf(g, x - e, y - e, z - e), v001 = box_sdf(g, x - e, y - e, z + e);
        float v010 = box_sdf(g, x - e, y + e, z - e), v011 = box_sdf(g, x - e, y + e, z + e);
        float v100 = box_sdf(g, x + e, y - e, z - e), v101 = box_sdf(g, x + e, y - e, z + e);
        float v110 = box_sdf(g, x + e, y + e, z - e), v111 = box_sdf(g, x + e, y + e, z + e);
        float gx = ((((v100 - v000) + (v101 - v001)) + (v110 - v010)) + (v111 - v011)) * 0.25f;
        float gy = ((((v010 - v000) + (v011 - v001)) + (v110 - v100)) + (v111 - v101)) * 0.25f;
        float gz = ((((v001 - v000) + (v011 - v010)) + (v101 - v100)) + (v111 - v110)) * 0.25f;
        float m2 = length2f(gx, gy, gz);
        if(m2 > FLT_MIN) {
            float s = sqrtf(m2);
            gx = gx / s; gy = gy / s; gz = gz / s;
            x = x - phiVal * gx;
            y = y - phiVal * gy;
            z = z - phiVal * gz;
        }
    }
}

// The same projection against every boundary group in turn (the static CSG union, then
// each dynamic object: the reference's moveParticles loops over m_BoundaryObjects,
// PIC_Solver.cpp:353-372); the domain box alone takes the path above.
__device__ __forceinline__ void constrain_particle(const GridDesc& g, float& x, float& y, float& z) {
    if(g.nObj == 0) {
        constrain_to_box(g, x, y, z);
        return;
    }
    const int ng = 1 + g.nObj - g.nStatic;
    for(int grp = 0; grp < ng; ++grp) {
        const float phiVal = group_sdf(g, grp, x, y, z);
        if(phiVal < 0.f) {
            const float e = 1e-4f;
            float v000 = group_sdf(g, grp, x - e, y - e, z - e), v001 = group_sdf(g, grp, x - e, y - e, z + e);
            float v010 = group_sdf(g, grp, x - e, y + e, z - e), v011 = group_sdf(g, grp, x - e, y + e, z + e);
            float v100 = group_sdf(g, grp, x + e, y - e, z - e), v101 = group_sdf(g, grp, x + e, y - e, z + e);
            float v110 = group_sdf(g, grp, x + e, y + e, z - e), v111 = group_sdf(g, grp, x + e, y + e, z + e);
            float gx = ((((v100 - v000) + (v101 - v001)) + (v110 - v010)) + (v111 - v011)) * 0.25f;
            float gy = ((((v010 - v000) + (v011 - v001)) + (v110 - v100)) + (v111 - v101)) * 0.25f;
            float gz = ((((v001 - v000) + (v011 - v010)) + (v101 - v100)) + (v111 - v110)) * 0.25f;
            float m2 = length2f(gx, gy, gz);
            if(m2 > FLT_MIN) {
                float s = sqrtf(m2);
                gx = gx / s; gy = gy / s; gz = gz / s;
                x = x - phiVal * gx;
                y = y - phiVal * gy;
                z = z - phiVal * gz;
            }
        }
    }
}

__device__ __forceinline__ uint32_t cell_linear(const GridDesc& g, float gx, float gy, float gz, bool& outside,
                                                int* cc = nullptr) {
    // Grid::getCellIdx<Int> (Grid.h:156-162): truncation of (p - bMin)/cellSize
    int c[3] = {(int)gx, (int)gy, (int)gz};
    outside = false;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        if(c[d] < 0) { c[d] = 0; outside = true; }
        if(c[d] > g.G[d] - 1) { c[d] = g.G[d] - 1; outside = true; }
    }
    if(cc) { cc[0] = c[0]; cc[1] = c[1]; cc[2] = c[2]; }
    return (uint32_t)(((size_t)c[2] * g.G[1] + c[1]) * g.G[0] + c[0]);
}

// Bounding box of occupied cells: per-thread box, reduced over the block, then one set
// of atomics per block (the advection grid is capped, so there are few blocks).
__device__ __forceinline__ void bbox_block_reduce(DevState* st, int mn[3], int mx[3]) {
    __shared__ int sm[2][3][32];
#pragma unroll
    for(int d = 0; d < 3; ++d)
        for(int off = 16; off > 0; off >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], off));
            mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], off));
        }
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if((threadIdx.x & 31) == 0) {
#pragma unroll
        for(int d = 0; d < 3; ++d) { sm[0][d][w] = mn[d]; sm[1][d][w] = mx[d]; }
    }
    __syncthreads();
    if(threadIdx.x < 3) {
        const int d = threadIdx.x;
        int a = INT_MAX, b = INT_MIN;
        for(int q = 0; q < nw; ++q) { a = min(a, sm[0][d][q]); b = max(b, sm[1][d][q]); }
        if(a != INT_MAX) atomicMin(&st->bbox[d], a);
        if(b != INT_MIN) atomicMax(&st->bbox[3 + d], b);
    }
}

// The block's box written to part[6 * bx ...] (min x,y,z, max x,y,z), no atomics
__device__ __forceinline__ void bbox_block_partial(int* __restrict__ part, unsigned bx, int mn[3], int mx[3]) {
    __shared__ int sm[2][3][32];
#pragma unroll
    for(int d = 0; d < 3; ++d)
        for(int off = 16; off > 0; off >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], off));
            mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], off));
        }
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if((threadIdx.x & 31) == 0) {
#pragma unroll
        for(int d = 0; d < 3; ++d) { sm[0][d][w] = mn[d]; sm[1][d][w] = mx[d]; }
    }
    __syncthreads();
    if(threadIdx.x < 3) {
        const int d = threadIdx.x;
        int a = INT_MAX, b = INT_MIN;
        for(int q = 0; q < nw; ++q) { a = min(a, sm[0][d][q]); b = max(b, sm[1][d][q]); }
        part[6 * bx + d] = a;
        part[6 * bx + 3 + d] = b;
    }
    __syncthreads();  // sm is free again (batched stages call this once per virtual block)
}

// Folds the per-block boxes into DevState::bbox
__device__ __forceinline__ void bbox_final_body(Blk blk, int nparts, const int* __restrict__ part, DevState* st) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for(int q = blk.x * blockDim.x + threadIdx.x; q < nparts; q += blk.n * blockDim.x) {
#pragma unroll
        for(int d = 0; d < 3; ++d) { mn[d] = min(mn[d], part[6 * q + d]); mx[d] = max(mx[d], part[6 * q + 3 + d]); }
    }
    bbox_block_reduce(st, mn, mx);
}
__global__ void __launch_bounds__(256) k_bbox_final(int nparts, const int* __restrict__ part, DevState* st) {
    bbox_final_body(own_blk(), nparts, part, st);
}

// ----------------------------------------------------------------------------------
// moveParticles + cell histogram
// ----------------------------------------------------------------------------------
// PIC_Solver::moveParticles (PIC_Solver.cpp:353-373) with trace_rk2 (:1137-1144), then the
// particle's cell id and its arrival slot in the cell histogram (the first half of the
// counting sort).
// Cell histogram slot of a particle with one atomic per cell and warp: lanes holding the
// same cell (most of a warp, the particles being in cell order from the last sort) take
// consecutive slots from their leader's atomicAdd.  The order of slots inside a cell is
// arbitrary either way: every bucket is sorted by particle id afterwards.  c = ~0u: no
// particle in this lane.  All 32 lanes of the warp must call it.
__device__ __forceinline__ void histogram_slot(uint32_t c, int p, uint32_t* __restrict__ count,
                                               uint32_t* __restrict__ slot) {
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    if(c == 0xffffffffu) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if(lane == leader) base = atomicAdd(count + c, (unsigned)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    slot[p] = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

__device__ __forceinline__ void advect_body(Blk blk, int n, float* __restrict__ px, float* __restrict__ py,
                                            float* __restrict__ pz, const float* __restrict__ u,
                                            const float* __restrict__ v, const float* __restrict__ w,
                                            const GridDesc& g, float sub, int steps, uint32_t* __restrict__ cellOf,
                                            uint32_t* __restrict__ slot, uint32_t* __restrict__ count, DevState* st,
                                            int* __restrict__ bboxPart) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    const int p = blk.x * blockDim.x + threadIdx.x;
    uint32_t c = 0xffffffffu;
    if(p < n) {
        float x = px[p], y = py[p], z = pz[p];
        for(int s = 0; s < steps; ++s) {
            float gv[3];
            float gx = (x - g.bmin[0]) / g.dx, gy = (y - g.bmin[1]) / g.dx, gz = (z - g.bmin[2]) / g.dx;
            vel_from_grid(g, u, v, w, gx, gy, gz, gv);
            const float h = 0.5f * sub;
            float mxp = x + h * gv[0], myp = y + h * gv[1], mzp = z + h * gv[2];
            gx = (mxp - g.bmin[0]) / g.dx; gy = (myp - g.bmin[1]) / g.dx; gz = (mzp - g.bmin[2]) / g.dx;
            vel_from_grid(g, u, v, w, gx, gy, gz, gv);
            x = x + sub * gv[0];
            y = y + sub * gv[1];
            z = z + sub * gv[2];
            constrain_particle(g, x, y, z);
        }
        px[p] = x; py[p] = y; pz[p] = z;
        bool outside;
        int cc[3];
        c = cell_linear(g, (x - g.bmin[0]) / g.dx, (y - g.bmin[1]) / g.dx, (z - g.bmin[2]) / g.dx, outside, cc);
        if(outside) atomicOr(&st->flags, BNN_FLAG_OUT_OF_GRID);
        cellOf[p] = c;
#pragma unroll
        for(int d = 0; d < 3; ++d) { mn[d] = cc[d]; mx[d] = cc[d]; }
    }
    histogram_slot(c, p, count, slot);
    bbox_block_partial(bboxPart, blk.x, mn, mx);
}
__global__ void __launch_bounds__(256, 6) k_advect(int n, float* __restrict__ px, float* __restrict__ py,
                                                float* __restrict__ pz, const float* __restrict__ u,
                                                const float* __restrict__ v, const float* __restrict__ w, GridDesc g,
                                                float sub, int steps, uint32_t* __restrict__ cellOf,
                                                uint32_t* __restrict__ slot, uint32_t* __restrict__ count,
                                                DevState* st, int* __restrict__ bboxPart) {
    advect_body(own_blk(), n, px, py, pz, u, v, w, g, sub, steps, cellOf, slot, count, st, bboxPart);
}

// ----------------------------------------------------------------------------------
// Position correction
// ----------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t smix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// PIC_Solver::correctParticlePositions (PIC_Solver.cpp:377-485), 3D, on the cell-sorted
// particles: springs to the other particles of the 3x3x3 cells (cells z, y, x major, a
// cell's particles in id order), MathHelpers::smooth_kernel with the cube rounded from
// the double product, a counter-based jitter (SplitMix64 over sub-step and the two
// particle ids, 21 bits per component) where two particles nearly coincide, then
// AdvectionSteps moves with the box projection.  Reads the old positions, writes `o`.
__global__ void __launch_bounds__(256) k_correct_positions(int n, GridDesc g, const float* __restrict__ px,
                                                           const float* __restrict__ py, const float* __restrict__ pz,
                                                           const uint32_t* __restrict__ ids,
                                                           const uint32_t* __restrict__ cellStart, float radius2,
                                                           float threshold2, float jitterScale, float kSpring,
                                                           int advSteps, unsigned long long step,
                                                           float* __restrict__ ox, float* __restrict__ oy,
                                                           float* __restrict__ oz) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const float x0 = px[p], y0 = py[p], z0 = pz[p];
    const int c[3] = {(int)((x0 - g.bmin[0]) / g.dx), (int)((y0 - g.bmin[1]) / g.dx), (int)((z0 - g.bmin[2]) / g.dx)};
    float sp[3] = {0.f, 0.f, 0.f};
    const uint32_t myId = ids[p];
    for(int dk = -1; dk <= 1; ++dk) {
        const int ck = c[2] + dk;
        if(ck < 0 || ck >= g.G[2]) continue;
        for(int dj = -1; dj <= 1; ++dj) {
            const int cj = c[1] + dj;
            if(cj < 0 || cj >= g.G[1]) continue;
            const int xlo = max(c[0] - 1, 0), xhi = min(c[0] + 1, g.G[0] - 1);
            if(xlo > xhi) continue;
            const size_t base = ((size_t)ck * g.G[1] + cj) * g.G[0];
            const uint32_t b = cellStart[base + xlo], e = cellStart[base + xhi + 1];
            for(uint32_t q = b; q < e; ++q) {
                if(q == (uint32_t)p) continue;
                const float dx = x0 - px[q], dy = y0 - py[q], dz = z0 - pz[q];
                const float d2 = length2f(dx, dy, dz);
                const float x2 = d2 / radius2;
                float w = 0.f;
                if(!(x2 > 1.0f)) {
                    const float t = 1.0f - x2;
                    w = (float)(((double)t * (double)t) * (double)t);
                }
                if(d2 > threshold2) {
                    const float s = sqrtf(d2);
                    sp[0] += w * dx / s;
                    sp[1] += w * dy / s;
                    sp[2] += w * dz / s;
                } else {
                    const uint64_t h = smix64(smix64(smix64((uint64_t)step) ^ (uint64_t)myId) ^ (uint64_t)ids[q]);
#pragma unroll
                    for(int a = 0; a < 3; ++a) {
                        const float u = (float)((h >> (21 * a)) & 0x1FFFFFull) * (1.0f / 2097152.0f);
                        sp[a] += jitterScale * (2.0f * u - 1.0f);
                    }
                }
            }
        }
    }
    float x = x0, y = y0, z = z0;
    for(int s = 0; s < advSteps; ++s) {
        x += sp[0] * kSpring;
        y += sp[1] * kSpring;
        z += sp[2] * kSpring;
        constrain_particle(g, x, y, z);
    }
    ox[p] = x; oy[p] = y; oz[p] = z;
}

// Cell id, histogram slot and the occupied-cell box of particles that were moved since the
// last sort (after position correction); grid-stride like k_advect
__global__ void __launch_bounds__(256) k_rebin(int n, const float* __restrict__ px, const float* __restrict__ py,
                                               const float* __restrict__ pz, GridDesc g,
                                               uint32_t* __restrict__ cellOf, uint32_t* __restrict__ slot,
                                               uint32_t* __restrict__ count, DevState* st) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    // the trip count is the same for the whole block (histogram_slot needs every lane)
    for(int p0 = blockIdx.x * blockDim.x; p0 < n; p0 += gridDim.x * blockDim.x) {
        const int p = p0 + threadIdx.x;
        uint32_t c = 0xffffffffu;
        if(p < n) {
            bool outside;
            int cc[3];
            c = cell_linear(g, (px[p] - g.bmin[0]) / g.dx, (py[p] - g.bmin[1]) / g.dx, (pz[p] - g.bmin[2]) / g.dx,
                            outside, cc);
            if(outside) atomicOr(&st->flags, BNN_FLAG_OUT_OF_GRID);
            cellOf[p] = c;
#pragma unroll
            for(int d = 0; d < 3; ++d) { mn[d] = min(mn[d], cc[d]); mx[d] = max(mx[d], cc[d]); }
        }
        histogram_slot(c, p, count, slot);
    }
    bbox_block_reduce(st, mn, mx);
}

__global__ void k_bbox_reset(DevState* st) {
    for(int d = 0; d < 3; ++d) { st->bbox[d] = INT_MAX; st->bbox[3 + d] = INT_MIN; }
}

// Cell id + histogram without moving (first sort of freshly loaded particles)
__global__ void k_cell_histogram(int n, const float* __restrict__ px, const float* __restrict__ py,
                                 const float* __restrict__ pz, GridDesc g, uint32_t* __restrict__ cellOf,
                                 uint32_t* __restrict__ slot, uint32_t* __restrict__ count, DevState* st) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    bool outside;
    uint32_t c = cell_linear(g, (px[p] - g.bmin[0]) / g.dx, (py[p] - g.bmin[1]) / g.dx, (pz[p] - g.bmin[2]) / g.dx,
                             outside);
    if(outside) atomicOr(&st->flags, BNN_FLAG_OUT_OF_GRID);
    cellOf[p] = c;
    slot[p] = atomicAdd(count + c, 1u);
}

// Counting-sort scatter: position of particle p = cellStart[cell] + arrival slot; the
// particle's id goes to the same position of key, so the bucket sort reads its keys
// contiguously instead of gathering them through order.
__device__ __forceinline__ void scatter_index_body(Blk blk, int n, const uint32_t* __restrict__ cellOf,
                                                   const uint32_t* __restrict__ slot,
                                                   const uint32_t* __restrict__ cellStart,
                                                   const uint32_t* __restrict__ ids, uint32_t* __restrict__ order,
                                                   uint32_t* __restrict__ key) {
    const int p = blk.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const uint32_t pos = cellStart[cellOf[p]] + slot[p];
    order[pos] = (uint32_t)p;
    key[pos] = ids[p];
}
__global__ void k_scatter_index(int n, const uint32_t* __restrict__ cellOf, const uint32_t* __restrict__ slot,
                                const uint32_t* __restrict__ cellStart, const uint32_t* __restrict__ ids,
                                uint32_t* __restrict__ order, uint32_t* __restrict__ key) {
    scatter_index_body(own_blk(), n, cellOf, slot, cellStart, ids, order, key);
}

// Arrival slots come from atomics, so each cell's bucket is put back into ascending
// particle-id order here: particles end up sorted by (cell, id), the order
// Grid::collectIndexToCells + getParticleIdxSortedByCell produce on one thread for
// particles stored in id order (Grid.cpp:92-114,299-309), whatever order they are stored
// in now.  The histogram is cleared for the next step on the way.
// Buckets of up to N particles are sorted in registers: both loads of the bucket are
// issued at once, then an odd-even transposition network (the ids are distinct, padding
// sorts last) puts them in order; larger buckets use an insertion sort in memory.
template<int N>
__device__ __forceinline__ void sort_bucket_regs(uint32_t* __restrict__ order, const uint32_t* __restrict__ key,
                                                 uint32_t b, uint32_t cnt) {
    uint32_t s[N], k[N];
#pragma unroll
    for(int q = 0; q < N; ++q) {
        s[q] = (uint32_t)q < cnt ? order[b + q] : 0u;
        k[q] = (uint32_t)q < cnt ? key[b + q] : 0xffffffffu;
    }
#pragma unroll
    for(int round = 0; round < N; ++round) {
#pragma unroll
        for(int q = round & 1; q + 1 < N; q += 2) {
            const bool sw = k[q] > k[q + 1];
            const uint32_t k0 = sw ? k[q + 1] : k[q], k1 = sw ? k[q] : k[q + 1];
            const uint32_t s0 = sw ? s[q + 1] : s[q], s1 = sw ? s[q] : s[q + 1];
            k[q] = k0; k[q + 1] = k1; s[q] = s0; s[q + 1] = s1;
        }
    }
#pragma unroll
    for(int q = 0; q < N; ++q)
        if((uint32_t)q < cnt) order[b + q] = s[q];
}

// Buckets of up to 16 particles are sorted in registers; larger ones (particles crowding
// into a cell, e.g. against a boundary) are listed for k_sort_large.
__device__ __forceinline__ void sort_buckets_body(Blk blk, int ncells, const uint32_t* __restrict__ cellStart,
                                                  uint32_t* __restrict__ order, const uint32_t* __restrict__ key,
                                                  uint32_t* __restrict__ count, uint32_t* __restrict__ largeList,
                                                  DevState* st) {
    const int c = blk.x * blockDim.x + threadIdx.x;
    if(c >= ncells) return;
    const uint32_t b = cellStart[c], e = cellStart[c + 1];
    count[c] = 0u;
    const uint32_t cnt = e - b;
    if(cnt < 2) return;
    if(cnt <= 8) { sort_bucket_regs<8>(order, key, b, cnt); return; }
    if(cnt <= 16) { sort_bucket_regs<16>(order, key, b, cnt); return; }
    largeList[atomicAdd(&st->nlarge, 1u)] = (uint32_t)c;
}
__global__ void __launch_bounds__(256, 6) k_sort_buckets(int ncells, const uint32_t* __restrict__ cellStart, uint32_t* __restrict__ order,
                               const uint32_t* __restrict__ key, uint32_t* __restrict__ count,
                               uint32_t* __restrict__ largeList, DevState* st) {
    sort_buckets_body(own_blk(), ncells, cellStart, order, key, count, largeList, st);
}

// One block per listed bucket: every particle's place is the number of particles of the
// bucket with a smaller id (ids are distinct), counted against keys staged in shared
// memory.  tmp[b, e) holds the bucket's unsorted order while it is rewritten.
__device__ __forceinline__ void sort_large_body(Blk blk, const uint32_t* __restrict__ cellStart,
                                                uint32_t* __restrict__ order, const uint32_t* __restrict__ ids,
                                                uint32_t* __restrict__ tmp, const uint32_t* __restrict__ largeList,
                                                const DevState* st) {
    __shared__ uint32_t sk[1024];
    const unsigned nl = st->nlarge;
    for(unsigned l = blk.x; l < nl; l += blk.n) {
        const uint32_t c = largeList[l];
        const uint32_t b = cellStart[c], cnt = cellStart[c + 1] - b;
        for(uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) tmp[b + i] = order[b + i];
        __syncthreads();
        for(uint32_t ib = 0; ib < cnt; ib += blockDim.x) {
            const uint32_t i = ib + threadIdx.x;
            const uint32_t v = i < cnt ? tmp[b + i] : 0u;
            const uint32_t key = i < cnt ? ids[v] : 0u;
            uint32_t rank = 0;
            for(uint32_t jb = 0; jb < cnt; jb += 1024) {
                const uint32_t m = min(1024u, cnt - jb);
                __syncthreads();
                for(uint32_t j = threadIdx.x; j < m; j += blockDim.x) sk[j] = ids[tmp[b + jb + j]];
                __syncthreads();
                for(uint32_t j = 0; j < m; ++j) rank += sk[j] < key ? 1u : 0u;
            }
            if(i < cnt) order[b + rank] = v;
        }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(256) k_sort_large(const uint32_t* __restrict__ cellStart, uint32_t* __restrict__ order,
                                                    const uint32_t* __restrict__ ids, uint32_t* __restrict__ tmp,
                                                    const uint32_t* __restrict__ largeList, const DevState* st) {
    sort_large_body(own_blk(), cellStart, order, ids, tmp, largeList, st);
}

// Apply the permutation to the particle arrays and emit what the gathers read per
// particle (all from Grid::getGridCoordinate, Grid.h:197):
//   rec  plane D < 3: the P2G stencil record of component D, {ex, ey, ez, v_D}: e_a is the
//        get_barycentric fraction of axis a (ArrayHelpers.h:95-112), its sign bit set when
//        the stencil's base index is the particle's (sort) cell - 1 instead of the cell
//        itself -- the only two cases, whatever the position, since both indices are
//        clamped the same way and fractions are never -0;
//        plane 3: the position {x, y, z, 0} for the fluid SDF.
// One 16-byte load per candidate particle then replaces four scattered 4-byte loads.
__device__ __forceinline__ void gather_particles_body(Blk blk, int n, const uint32_t* __restrict__ order,
                                                      const float* __restrict__ src6, const float* __restrict__ srcPos,
                                                      float* __restrict__ dst6, const uint32_t* __restrict__ idSrc,
                                                      uint32_t* __restrict__ idDst, const float* __restrict__ cSrc,
                                                      float* __restrict__ cDst, float4* __restrict__ rec,
                                                      const GridDesc& g, size_t stride) {
    const int i = blk.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const uint32_t s = order[i];
    float v6[6];
    // positions from srcPos when the move wrote them apart (k_g2p_move), else from src6
#pragma unroll
    for(int q = 0; q < 6; ++q) {
        v6[q] = q < 3 ? srcPos[q * stride + s] : src6[q * stride + s];
        dst6[q * stride + i] = v6[q];
    }
    idDst[i] = idSrc[s];
    float gc[3];
#pragma unroll
    for(int a = 0; a < 3; ++a) gc[a] = (v6[a] - g.bmin[a]) / g.dx;
    if(cSrc) {
#pragma unroll
        for(int q = 0; q < 9; ++q) cDst[q * stride + i] = cSrc[q * stride + s];
    }
    rec[3 * stride + i] = make_float4(v6[0], v6[1], v6[2], 0.f);
    int cell[3];
#pragma unroll
    for(int a = 0; a < 3; ++a) {
        int c = (int)gc[a];
        cell[a] = c < 0 ? 0 : (c > g.G[a] - 1 ? g.G[a] - 1 : c);
    }
#pragma unroll
    for(int D = 0; D < 3; ++D) {
        float e[3];
#pragma unroll
        for(int a = 0; a < 3; ++a) {
            int si;
            float fi;
            bary(gc[a] - (a == D ? 0.f : 0.5f), si, fi, g.G[a] + (a == D ? 1 : 0));
            e[a] = (si < cell[a]) ? __int_as_float(__float_as_int(fi) | (int)0x80000000) : fi;
        }
        rec[D * stride + i] = make_float4(e[0], e[1], e[2], v6[3 + D]);
    }
}
__global__ void k_gather_particles(int n, const uint32_t* __restrict__ order, const float* __restrict__ src6,
                                   const float* __restrict__ srcPos, float* __restrict__ dst6,
                                   const uint32_t* __restrict__ idSrc, uint32_t* __restrict__ idDst,
                                   const float* __restrict__ cSrc, float* __restrict__ cDst,
                                   float4* __restrict__ rec, GridDesc g, size_t stride) {
    gather_particles_body(own_blk(), n, order, src6, srcPos, dst6, idSrc, idDst, cSrc, cDst, rec, g, stride);
}

// ----------------------------------------------------------------------------------
// PIC grid advection
// ----------------------------------------------------------------------------------
// PIC_Solver::advectGridVelocity + trace_rk2_grid (PIC_Solver.cpp:489-501, 1148-1154) for
// component D: every face is traced back by RK2 through the grid velocity in grid units
// (velocity x invCellSize) and takes component D there.  The caller swaps the output in
// before the next component, as the reference copies each component back in turn.
template<int D>
__global__ void __launch_bounds__(256) k_advect_grid(GridDesc g, const float* __restrict__ u,
                                                     const float* __restrict__ v, const float* __restrict__ w,
                                                     float inv, float dt, float* __restrict__ out) {
    const int sx = g.G[0] + (D == 0), sy = g.G[1] + (D == 1), sz = g.G[2] + (D == 2);
    const size_t nf = (size_t)sx * sy * sz;
    const size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(f >= nf) return;
    const int i = (int)(f % sx);
    const int j = (int)((f / sx) % sy);
    const int k = (int)(f / ((size_t)sx * sy));
    const float ts = -dt;
    const float gp[3] = {(float)i + (D == 0 ? 0.f : 0.5f), (float)j + (D == 1 ? 0.f : 0.5f),
                         (float)k + (D == 2 ? 0.f : 0.5f)};
    float gv[3];
    vel_from_grid(g, u, v, w, gp[0], gp[1], gp[2], gv);
    for(int c = 0; c < 3; ++c) gv[c] = gv[c] * inv;
    const float h = 0.5f * ts;
    const float mid[3] = {gp[0] + h * gv[0], gp[1] + h * gv[1], gp[2] + h * gv[2]};
    vel_from_grid(g, u, v, w, mid[0], mid[1], mid[2], gv);
    for(int c = 0; c < 3; ++c) gv[c] = gv[c] * inv;
    const float bx = gp[0] + ts * gv[0], by = gp[1] + ts * gv[1], bz = gp[2] + ts * gv[2];
    float val;
    if(D == 0) val = interp_face(u, sx, sy, sz, bx, by - 0.5f, bz - 0.5f);
    else if(D == 1) val = interp_face(v, sx, sy, sz, bx - 0.5f, by, bz - 0.5f);
    else val = interp_face(w, sx, sy, sz, bx - 0.5f, by - 0.5f, bz);
    out[f] = val;
}

// ----------------------------------------------------------------------------------
// Velocity extrapolation (one layer)
// ----------------------------------------------------------------------------------
// Face-index distance (Chebyshev, per axis beyond the box) of face (i,j,k) from the
// occupied-cell bounding box; INT_MAX when there are no particles.  Faces of any component
// that P2G or the pressure update make valid lie within distance 2: P2G reaches faces
// c-1..c+1 of a particle's cell c, fluid cells (phi < 0) lie within one cell of a
// particle, and a face touches the cells a and a-1 on its own axis.
__device__ __forceinline__ int bbox_distance(const DevState* st, int i, int j, int k) {
    const int c[3] = {i, j, k};
    int o = 0;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const int lo = st->bbox[d], hi = st->bbox[3 + d];
        if(hi < lo) return INT_MAX;
        o = max(o, max(lo - c[d], c[d] - hi));
    }
    return o;
}
// Each extrapolation layer makes valid only faces next to valid ones, so after 4 layers
// every valid face is within kExtFull of the box and faces farther than that never
// change.  Layers therefore compute faces up to kExtFull, copy those up to kExtRegion
// (the neighbours the computed faces read, kept defined in both ping-pong buffers) and
// leave the rest alone: there the input is 0 and invalid and stays so.
constexpr int kExtFull = 2 + 4;
constexpr int kExtRegion = kExtFull + 2;

// The box of faces within `reach` of the occupied-cell box, clamped to an array of size
// S; false when it is empty (no particles).
__device__ __forceinline__ bool reach_box(const DevState* st, int reach, const int S[3], int lo[3], int hi[3]) {
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const int bl = st->bbox[d], bh = st->bbox[3 + d];
        if(bh < bl) return false;
        lo[d] = max(bl - reach, 0);
        hi[d] = min(bh + reach, S[d] - 1);
        if(hi[d] < lo[d]) return false;
    }
    return true;
}

// One layer of PIC_Solver::extrapolateVelocity (PIC_Solver.cpp:998-1089): an interior
// face that was not valid takes the mean of its valid 6-neighbours (+x,-x,+y,-y,+z,-z
// summation order) and becomes valid; everything reads the previous layer.
// mode 0: plain layer.  mode 1 (last layer after P2G): also writes the FLIP backup
// oldVels (FLIP_Data.h:48-52) and applies Earth gravity v -= 9.81*dt (PIC_Solver.cpp:
// 505-511) to the v component; beyond the region the host has already written the
// backup 0 and the velocity 0 - gravityDt.  mode 2 (last layer after projection): folds
// max|u| into the CFL reduction (PIC_Solver.cpp:342-349).
// The blocks stride over tiles of 8 rows of the region boxes only.
// The three components go through a layer in one launch: their region tiles form one
// index space (32-bit tile arithmetic), so the small per-component regions fill the GPU
// together.
struct ExtLayer {
    const float* gin[3];
    const uint8_t* vin[3];
    float* gout[3];
    uint8_t* vout[3];
    float* oldOut[3];
    float gdt[3];
    int S[3][3];
    int mode;
};

// The region box of component D (faces within kExtRegion of the occupied-cell box bb,
// clamped to the array; reach_box) and its tile count: tiles are 8 rows (j) of one k plane.
template<int D>
__device__ __forceinline__ unsigned ext_box(const ExtLayer& a, const int bb[6], int lo[3], int hi[3], unsigned& ty) {
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        lo[d] = max(bb[d] - kExtRegion, 0);
        hi[d] = min(bb[3 + d] + kExtRegion, a.S[D][d] - 1);
        if(hi[d] < lo[d]) { ty = 1; return 0u; }
    }
    ty = (unsigned)(hi[1] - lo[1] + 8) / 8;
    return ty * (unsigned)(hi[2] - lo[2] + 1);
}

// One tile, each of its rows walked along x by one warp; returns max |value| written.
template<int D>
__device__ __forceinline__ float ext_tile(const ExtLayer& a, unsigned t, const int bb[6]) {
    int lo[3], hi[3];
    unsigned ty;
    ext_box<D>(a, bb, lo, hi, ty);
    const int sx = a.S[D][0], sy = a.S[D][1], sz = a.S[D][2];
    const int j = lo[1] + (int)(t % ty) * 8 + (int)(threadIdx.x >> 5);
    const int k = lo[2] + (int)(t / ty);
    if(j > hi[1]) return 0.f;
    const float* __restrict__ gin = a.gin[D];
    const uint8_t* __restrict__ vin = a.vin[D];
    const size_t sxy = (size_t)sx * sy;
    const size_t rowBase = ((size_t)k * sy + j) * sx;
    // bbox_distance split: the row's distance along y and z, then x per face
    const int ojk = max(max(max(bb[1] - j, j - bb[4]), max(bb[2] - k, k - bb[5])), 0);
    const bool interiorJK = j > 0 && j < sy - 1 && k > 0 && k < sz - 1;
    float m = 0.f;
    for(int i = lo[0] + (int)(threadIdx.x & 31); i <= hi[0]; i += 32) {
        const size_t f = rowBase + i;
        const int o = max(ojk, max(bb[0] - i, i - bb[3]));
        float val = gin[f];
        uint8_t vv = vin[f];
        if(!vv && o <= kExtFull && interiorJK && i > 0 && i < sx - 1) {
            float sum = 0.f;
            unsigned count = 0;
            if(vin[f + 1]) { sum += gin[f + 1]; ++count; }
            if(vin[f - 1]) { sum += gin[f - 1]; ++count; }
            if(vin[f + sx]) { sum += gin[f + sx]; ++count; }
            if(vin[f - sx]) { sum += gin[f - sx]; ++count; }
            if(vin[f + sxy]) { sum += gin[f + sxy]; ++count; }
            if(vin[f - sxy]) { sum += gin[f - sxy]; ++count; }
            if(count > 0) { val = sum / (float)count; vv = 2; }  // 2: extrapolated in this pass
        }
        a.vout[D][f] = vv;
        if(a.mode == 1) {
            a.oldOut[D][f] = val;
            a.gout[D][f] = val - a.gdt[D];
        } else {
            a.gout[D][f] = val;
        }
        m = fmaxf(m, fabsf(val));
    }
    return m;
}

__device__ __forceinline__ void extrapolate3_body(Blk blk, const ExtLayer& a, DevState* st) {
    int bb[6];
#pragma unroll
    for(int q = 0; q < 6; ++q) bb[q] = st->bbox[q];
    float m = 0.f;
    if(bb[3] >= bb[0]) {  // no particles: nothing changes
        unsigned n0, n1, n2;
        {
            int lo[3], hi[3];
            unsigned ty;
            n0 = ext_box<0>(a, bb, lo, hi, ty);
            n1 = ext_box<1>(a, bb, lo, hi, ty);
            n2 = ext_box<2>(a, bb, lo, hi, ty);
        }
        const unsigned n01 = n0 + n1, total = n01 + n2;
        for(unsigned t = blk.x; t < total; t += blk.n) {
            float v;
            if(t < n0) v = ext_tile<0>(a, t, bb);
            else if(t < n01) v = ext_tile<1>(a, t - n0, bb);
            else v = ext_tile<2>(a, t - n01, bb);
            m = fmaxf(m, v);
        }
    }
    if(a.mode == 2) {
        __shared__ float sm[8];
        for(int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
        if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
        __syncthreads();
        if(threadIdx.x == 0) {
            for(int w = 1; w < 8; ++w) m = fmaxf(m, sm[w]);
            if(m > 0.f) atomicMax(&st->maxvel_bits, __float_as_uint(m));
        }
    }
}
__global__ void __launch_bounds__(256, 8) k_extrapolate3(ExtLayer a, DevState* st) { extrapolate3_body(own_blk(), a, st); }

// max |a| over an array, folded into *maxBits (float bits of a non-negative value order
// like the unsigned integers)
__global__ void __launch_bounds__(256) k_maxabs(const float* __restrict__ a, size_t n, unsigned* maxBits) {
    float m = 0.f;
    for(size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(a[i]));
    __shared__ float sm[8];
    for(int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if(threadIdx.x == 0) {
        for(int w = 1; w < 8; ++w) m = fmaxf(m, sm[w]);
        if(m > 0.f) atomicMax(maxBits, __float_as_uint(m));
    }
}

__device__ __forceinline__ void fill_body(Blk blk, float* __restrict__ a, size_t n, float v) {
    for(size_t i = (size_t)blk.x * blockDim.x + threadIdx.x; i < n; i += (size_t)blk.n * blockDim.x) a[i] = v;
}
__global__ void k_fill(float* __restrict__ a, size_t n, float v) { fill_body(own_blk(), a, n, v); }

// ----------------------------------------------------------------------------------
// Pressure system
// ----------------------------------------------------------------------------------
// Active-cell flags for PIC_Solver::computeSystem's numbering loop (PIC_Solver.cpp:706-712)
__device__ __forceinline__ void active_flags_body(Blk blk, const GridDesc& g, const float* __restrict__ phi,
                                                  uint32_t* __restrict__ flag, DevState* st) {
    const size_t nc = (size_t)g.G[0] * g.G[1] * g.G[2];
    const size_t c = (size_t)blk.x * blockDim.x + threadIdx.x;
    if(c >= nc) return;
    const float p = phi[c];
    flag[c] = p < 0.f ? 1u : 0u;
    if(p == 0.f) {
        const int i = (int)(c % g.G[0]);
        const int j = (int)((c / g.G[0]) % g.G[1]);
        const int k = (int)(c / ((size_t)g.G[0] * g.G[1]));
        if(i > 0 && i < g.G[0] - 1 && j > 0 && j < g.G[1] - 1 && k > 0 && k < g.G[2] - 1) atomicAdd(&st->zero_phi, 1u);
    }
}
__global__ void k_active_flags(GridDesc g, const float* __restrict__ phi, uint32_t* __restrict__ flag,
                               DevState* st) {
    active_flags_body(own_blk(), g, phi, flag, st);
}

__device__ __forceinline__ void active_rows_body(Blk blk, size_t nc, const uint32_t* __restrict__ flag,
                                                 const uint32_t* __restrict__ idx, uint32_t* __restrict__ rowCell) {
    const size_t c = (size_t)blk.x * blockDim.x + threadIdx.x;
    if(c >= nc) return;
    if(flag[c]) rowCell[idx[c]] = (uint32_t)c;
}
__global__ void k_active_rows(size_t nc, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ idx,
                              uint32_t* __restrict__ rowCell) {
    active_rows_body(own_blk(), nc, flag, idx, rowCell);
}

// One row of PIC_Solver::computeSystem (PIC_Solver.cpp:794-891) for a static scene
// (face weights 1): rhs = -div u, diagonal accumulated in the order right, left, top,
// bottom, far, near with the ghost-fluid 1/theta terms, neighbour rows for fluid
// neighbours.  Neighbours are stored in ascending column order (-z,-y,-x,+x,+y,+z), the
// order FixedSparseMatrix::multiply sums them in (SparseMatrix.cpp:222-235).
template<bool WEIGHTED>
__device__ __forceinline__ void build_rows_body(Blk blk, const GridDesc& g, int nrows, const uint32_t* __restrict__ rowCell,
                                                const float* __restrict__ phi, const uint32_t* __restrict__ aidx,
                                                const float* __restrict__ u, const float* __restrict__ v,
                                                const float* __restrict__ w, const float* __restrict__ wu,
                                                const float* __restrict__ wv, const float* __restrict__ ww, float dt,
                                                float* __restrict__ rhs, float* __restrict__ diag,
                                                float* __restrict__ invdiag, int32_t* __restrict__ nbr,
                                                float* __restrict__ coef, DevState* st) {
    const int r = blk.x * blockDim.x + threadIdx.x;
    if(r >= nrows) return;
    const uint32_t c = rowCell[r];
    const int G0 = g.G[0], G1 = g.G[1], G2 = g.G[2];
    const int i = (int)(c % G0);
    const int j = (int)((c / G0) % G1);
    const int k = (int)(c / ((size_t)G0 * G1));
    int32_t nb[6] = {-1, -1, -1, -1, -1, -1};
    if(i < 1 || i > G0 - 2 || j < 1 || j > G1 - 2 || k < 1 || k > G2 - 2) {
        // fluid in the outer cell ring: the reference numbers it but never writes its row
        atomicOr(&st->flags, BNN_FLAG_RING_FLUID);
        rhs[r] = 0.f; diag[r] = 0.f; invdiag[r] = 0.f;
#pragma unroll
        for(int q = 0; q < 6; ++q) nbr[(size_t)q * nrows + r] = -1;
        if(WEIGHTED)
#pragma unroll
            for(int q = 0; q < 6; ++q) coef[(size_t)q * nrows + r] = 0.f;
        return;
    }
    const size_t sxu = G0 + 1, sxv = G0, sxw = G0;
    const size_t sxyu = sxu * G1, sxyv = (size_t)G0 * (G1 + 1), sxyw = (size_t)G0 * G1;
    const float pc = phi[c];
    const size_t GG = (size_t)G0 * G1;
    const float pr = phi[c + 1], pl = phi[c - 1], pt = phi[c + G0], pb = phi[c - G0], pf = phi[c + GG], pn = phi[c - GG];
    // faces: right, left, top, bottom, far, near
    const size_t fidx[6] = {(size_t)k * sxyu + (size_t)j * sxu + i + 1, (size_t)k * sxyu + (size_t)j * sxu + i,
                            (size_t)k * sxyv + (size_t)(j + 1) * sxv + i, (size_t)k * sxyv + (size_t)j * sxv + i,
                            (size_t)(k + 1) * sxyw + (size_t)j * sxw + i, (size_t)k * sxyw + (size_t)j * sxw + i};
    float wt[6] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f};
    if(WEIGHTED) {
        wt[0] = wu[fidx[0]]; wt[1] = wu[fidx[1]]; wt[2] = wv[fidx[2]];
        wt[3] = wv[fidx[3]]; wt[4] = ww[fidx[4]]; wt[5] = ww[fidx[5]];
    }
    float rv = 0.f;
    rv -= wt[0] * u[fidx[0]];
    rv += wt[1] * u[fidx[1]];
    rv -= wt[2] * v[fidx[2]];
    rv += wt[3] * v[fidx[3]];
    rv -= wt[4] * w[fidx[4]];
    rv += wt[5] * w[fidx[5]];
    rhs[r] = rv;
    float center = 0.f;
    const float phn[6] = {pr, pl, pt, pb, pf, pn};
    const size_t nc_[6] = {c + 1, c - 1, c + G0, c - G0, c + GG, c - GG};
    const int slotOf[6] = {3, 2, 4, 1, 5, 0};
    float co[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for(int q = 0; q < 6; ++q) {
        const float term = wt[q] * dt;
        if(phn[q] < 0.f) {
            center += term;
            nb[slotOf[q]] = (int32_t)aidx[nc_[q]];
            co[slotOf[q]] = -term;
        } else {
            const float th = smax(0.01f, fraction_inside(pc, phn[q]));
            center += term / th;
        }
    }
    diag[r] = center;
    // a cell closed off by zero-weight (solid) faces has a zero diagonal: Jacobi weight 0
    invdiag[r] = center != 0.f ? 1.0f / center : 0.f;
#pragma unroll
    for(int q = 0; q < 6; ++q) nbr[(size_t)q * nrows + r] = nb[q];
    if(WEIGHTED)
#pragma unroll
        for(int q = 0; q < 6; ++q) coef[(size_t)q * nrows + r] = co[q];
}
template<bool WEIGHTED>
__global__ void k_build_rows(GridDesc g, int nrows, const uint32_t* __restrict__ rowCell,
                             const float* __restrict__ phi, const uint32_t* __restrict__ aidx,
                             const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                             const float* __restrict__ wu, const float* __restrict__ wv, const float* __restrict__ ww,
                             float dt, float* __restrict__ rhs, float* __restrict__ diag, float* __restrict__ invdiag,
                             int32_t* __restrict__ nbr, float* __restrict__ coef, DevState* st) {
    build_rows_body<WEIGHTED>(own_blk(), g, nrows, rowCell, phi, aidx, u, v, w, wu, wv, ww, dt, rhs, diag, invdiag, nbr,
                              coef, st);
}

// ----------------------------------------------------------------------------------
// Pressure update
// ----------------------------------------------------------------------------------
// PIC_Solver::updateProjectedVelocity (PIC_Solver.cpp:911-981): face (i,j,k) of component
// D between cells c- and c gets u -= dt*(p_c - p_c-)/max(0.01, theta) when either cell is
// fluid and the face weight is positive (weights 1 without solid boundaries), and is
// marked valid; every other face is set to 0.  Fluid cells lie
// within one cell of the occupied-cell box, so only faces within 2 of it can be valid:
// the blocks stride over that box and the host zeroes the output arrays beforehand.
template<int D>
__device__ __forceinline__ void update_velocity_body(Blk blk, const GridDesc& g, const DevState* __restrict__ st,
                                                     const float* __restrict__ phi, const uint32_t* __restrict__ aidx,
                                                     const float* __restrict__ pressure, float dt,
                                                     const float* __restrict__ velIn, float* __restrict__ velOut,
                                                     uint8_t* __restrict__ validOut, const float* __restrict__ weight) {
    const int S[3] = {g.G[0] + (D == 0), g.G[1] + (D == 1), g.G[2] + (D == 2)};
    int lo[3], hi[3];
    if(!reach_box(st, 2, S, lo, hi)) return;
    // tiles of 8 rows (j) of one k plane; a warp walks its row along x
    const unsigned ty = (unsigned)(hi[1] - lo[1] + 8) / 8, nt = ty * (unsigned)(hi[2] - lo[2] + 1);
    const int amax = g.G[D];
    const size_t step = D == 0 ? 1 : (D == 1 ? (size_t)g.G[0] : (size_t)g.G[0] * g.G[1]);
    for(unsigned t = blk.x; t < nt; t += blk.n) {
        const int j = lo[1] + (int)(t % ty) * 8 + (int)(threadIdx.x >> 5);
        const int k = lo[2] + (int)(t / ty);
        if(j > hi[1]) continue;
        const size_t fRow = ((size_t)k * S[1] + j) * S[0];
        const size_t cRow = ((size_t)k * g.G[1] + j) * g.G[0];
        for(int i = lo[0] + (int)(threadIdx.x & 31); i <= hi[0]; i += 32) {
            const size_t f = fRow + i;
            const int a = D == 0 ? i : (D == 1 ? j : k);
            float out = 0.f;
            uint8_t vv = 0;
            if(a > 0 && a < amax) {
                const size_t c = cRow + i;
                const size_t cm = c - step;
                const float pc = phi[c], pm = phi[cm];
                if((pc < 0.f || pm < 0.f) && (!weight || weight[f] > 0.f)) {
                    const float prc = pc < 0.f ? pressure[aidx[c]] : 0.f;
                    const float prm = pm < 0.f ? pressure[aidx[cm]] : 0.f;
                    const float th = smax(0.01f, fraction_inside(pm, pc));
                    out = velIn[f] - dt * (prc - prm) / th;
                    vv = 1;
                }
            }
            velOut[f] = out;
            validOut[f] = vv;
        }
    }
}
template<int D>
__global__ void __launch_bounds__(256) k_update_velocity(GridDesc g, const DevState* __restrict__ st,
                                                         const float* __restrict__ phi,
                                                         const uint32_t* __restrict__ aidx,
                                                         const float* __restrict__ pressure, float dt,
                                                         const float* __restrict__ velIn, float* __restrict__ velOut,
                                                         uint8_t* __restrict__ validOut,
                                                         const float* __restrict__ weight) {
    update_velocity_body<D>(own_blk(), g, st, phi, aidx, pressure, dt, velIn, velOut, validOut, weight);
}

// ----------------------------------------------------------------------------------
// Solid boundaries (dynamic boundary objects)
// ----------------------------------------------------------------------------------
// MathHelpers::fraction_inside(bl, br, tl, tr) (MathHelpers.h:821-900), the area fraction
// of a square whose corners have these signed distances that lies inside (negative); the
// corners are walked as the cycle bl, br, tr, tl, rotated to a canonical start.
__device__ __forceinline__ float fraction_inside4(float bl, float br, float tl, float tr) {
    const int inside = (bl < 0.f ? 1 : 0) + (tl < 0.f ? 1 : 0) + (br < 0.f ? 1 : 0) + (tr < 0.f ? 1 : 0);
    float l[4] = {bl, br, tr, tl};
    auto rotate = [&l]() { const float t = l[0]; l[0] = l[1]; l[1] = l[2]; l[2] = l[3]; l[3] = t; };
    if(inside == 4) return 1.0f;
    if(inside == 3) {
        for(int it = 0; it < 4 && l[0] < 0.f; ++it) rotate();
        const float side0 = 1.0f - fraction_inside(l[0], l[3]);
        const float side1 = 1.0f - fraction_inside(l[0], l[1]);
        return 1.0f - 0.5f * side0 * side1;
    }
    if(inside == 2) {
        for(int it = 0; it < 4 && (l[0] >= 0.f || !(l[1] < 0.f || l[2] < 0.f)); ++it) rotate();
        if(l[1] < 0.f) {
            const float left = fraction_inside(l[0], l[3]);
            const float right = fraction_inside(l[1], l[2]);
            return 0.5f * (left + right);
        }
        const float mid = 0.25f * (l[0] + l[1] + l[2] + l[3]);
        if(mid < 0.f) {
            float area = 0.f;
            const float side1 = 1.0f - fraction_inside(l[0], l[3]);
            const float side3 = 1.0f - fraction_inside(l[2], l[3]);
            area += 0.5f * side1 * side3;
            const float side2 = 1.0f - fraction_inside(l[2], l[1]);
            const float side0 = 1.0f - fraction_inside(l[0], l[1]);
            area += 0.5f * side0 * side2;
            return 1.0f - area;
        }
        float area = 0.f;
        const float side0 = fraction_inside(l[0], l[1]);
        const float side1 = fraction_inside(l[0], l[3]);
        area += 0.5f * side0 * side1;
        const float side2 = fraction_inside(l[2], l[1]);
        const float side3 = fraction_inside(l[2], l[3]);
        area += 0.5f * side2 * side3;
        return area;
    }
    if(inside == 1) {
        for(int it = 0; it < 4 && l[0] >= 0.f; ++it) rotate();
        const float side0 = fraction_inside(l[0], l[3]);
        const float side1 = fraction_inside(l[0], l[1]);
        return 0.5f * side0 * side1;
    }
    return 0.f;
}

// PIC_Solver::computeBoundarySDF (PIC_Solver.cpp:1157-1168): at every grid node the
// minimum over the boundary objects (the static CSG union first, then the dynamic ones)
__global__ void k_node_sdf(GridDesc g, float* __restrict__ out) {
    const int nx = g.G[0] + 1, ny = g.G[1] + 1, nz = g.G[2] + 1;
    const size_t total = (size_t)nx * ny * nz;
    const int ng = 1 + g.nObj - g.nStatic;
    for(size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((size_t)nx * ny));
        const float x = g.bmin[0] + (float)i * g.dx, y = g.bmin[1] + (float)j * g.dx, z = g.bmin[2] + (float)k * g.dx;
        float m = 3.402823466e+38f;
        for(int grp = 0; grp < ng; ++grp) m = smin(m, group_sdf(g, grp, x, y, z));
        out[t] = m;
    }
}

// PIC_Solver::computeCellWeights (PIC_Solver.cpp:565-597): weight of a face = the part of
// it outside the solid, 1 - fraction_inside of its four corner nodes, clamped to [0, 1]
template<int D>
__global__ void k_face_weights(GridDesc g, const float* __restrict__ nsdf, float* __restrict__ wout) {
    const int sx = g.G[0] + (D == 0), sy = g.G[1] + (D == 1), sz = g.G[2] + (D == 2);
    const int nx = g.G[0] + 1, ny = g.G[1] + 1;
    const size_t total = (size_t)sx * sy * sz;
    for(size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % sx), j = (int)((t / sx) % sy), k = (int)(t / ((size_t)sx * sy));
        auto N = [&](int a, int b, int c) { return nsdf[((size_t)c * ny + b) * nx + a]; };
        float f;
        if(D == 0) f = fraction_inside4(N(i, j, k), N(i, j + 1, k), N(i, j, k + 1), N(i, j + 1, k + 1));
        else if(D == 1) f = fraction_inside4(N(i, j, k), N(i, j, k + 1), N(i + 1, j, k), N(i + 1, j, k + 1));
        else f = fraction_inside4(N(i, j, k), N(i, j + 1, k), N(i + 1, j, k), N(i + 1, j + 1, k));
        const float tmp = 1.0f - f;
        wout[t] = tmp < 0.f ? 0.f : (tmp > 1.0f ? 1.0f : tmp);  // MathHelpers::clamp01
    }
}

// PIC_Solver::computeFluidSDF, solid part (PIC_Solver.cpp:671-688): a cell near the fluid
// (phi < dx/2) whose corners average to inside the solid becomes fluid at -dx/2
__global__ void k_solid_extend(GridDesc g, const float* __restrict__ nsdf, float* __restrict__ phi) {
    const int nx = g.G[0] + 1, ny = g.G[1] + 1;
    const size_t total = (size_t)g.G[0] * g.G[1] * g.G[2];
    const float half = 0.5f * g.dx;
    for(size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        if(!(phi[t] < half)) continue;
        const int i = (int)(t % g.G[0]), j = (int)((t / g.G[0]) % g.G[1]), k = (int)(t / ((size_t)g.G[0] * g.G[1]));
        auto N = [&](int a, int b, int c) { return nsdf[((size_t)c * ny + b) * nx + a]; };
        const float solid = 0.125f * (N(i, j, k) + N(i + 1, j, k) + N(i, j + 1, k) + N(i + 1, j + 1, k) +
                                      N(i, j, k + 1) + N(i + 1, j, k + 1) + N(i, j + 1, k + 1) + N(i + 1, j + 1, k + 1));
        if(solid < 0.f) phi[t] = -half;
    }
}

// ArrayHelpers::interpolateGradient 3D (ArrayHelpers.cpp:214-251) of the node SDF
__device__ __forceinline__ void node_gradient(const float* __restrict__ a, int nx, int ny, int nz, float px, float py,
                                              float pz, float out[3]) {
    int i, j, k;
    float fi, fj, fk;
    bary(px, i, fi, nx);
    bary(py, j, fj, ny);
    bary(pz, k, fk, nz);
    auto A = [&](int x, int y, int z) { return a[((size_t)z * ny + y) * nx + x]; };
    const float v000 = A(i, j, k), v001 = A(i, j, k + 1), v010 = A(i, j + 1, k), v011 = A(i, j + 1, k + 1);
    const float v100 = A(i + 1, j, k), v101 = A(i + 1, j, k + 1), v110 = A(i + 1, j + 1, k), v111 = A(i + 1, j + 1, k + 1);
    // MathHelpers::bilerp(v00, v10, v01, v11, fx, fy) = lerp(lerp(v00, v10, fx), lerp(v01, v11, fx), fy)
    auto bil = [](float v00, float v10, float v01, float v11, float fx, float fy) {
        return lerpf(lerpf(v00, v10, fx), lerpf(v01, v11, fx), fy);
    };
    out[0] = bil(v100 - v000, v110 - v010, v101 - v001, v111 - v011, fj, fk);
    out[1] = bil(v010 - v000, v110 - v100, v011 - v001, v111 - v101, fi, fk);
    out[2] = bil(v001 - v000, v101 - v100, v011 - v010, v111 - v110, fi, fj);
}

// PIC_Solver::constrainGridVelocity (PIC_Solver.cpp:1093-1115), component D: a face that
// the last extrapolation filled (valid flag 2) and whose weight is 0 loses the velocity
// component along the boundary normal.  The new values go to tmp (candidate faces only)
// and are copied back by k_constrain_apply, so every face reads the component as it was.
template<int D>
__global__ void __launch_bounds__(256) k_constrain_compute(GridDesc g, const DevState* __restrict__ st,
                                                           const float* __restrict__ u, const float* __restrict__ v,
                                                           const float* __restrict__ w,
                                                           const uint8_t* __restrict__ valid,
                                                           const float* __restrict__ weight,
                                                           const float* __restrict__ nsdf, float* __restrict__ tmp) {
    const int S[3] = {g.G[0] + (D == 0), g.G[1] + (D == 1), g.G[2] + (D == 2)};
    int lo[3], hi[3];
    if(!reach_box(st, kExtFull, S, lo, hi)) return;
    const long long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    for(long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nx * ny * nz;
        t += (long long)gridDim.x * blockDim.x) {
        const int i = lo[0] + (int)(t % nx), j = lo[1] + (int)((t / nx) % ny), k = lo[2] + (int)(t / (nx * ny));
        const size_t f = ((size_t)k * S[1] + j) * S[0] + i;
        if(valid[f] != 2 || !(weight[f] < FLT_MIN)) continue;
        const float gp[3] = {(float)i + (D == 0 ? 0.f : 0.5f), (float)j + (D == 1 ? 0.f : 0.5f),
                             (float)k + (D == 2 ? 0.f : 0.5f)};
        float vel[3];
        vel_from_grid(g, u, v, w, gp[0], gp[1], gp[2], vel);
        float nrm[3];
        node_gradient(nsdf, g.G[0] + 1, g.G[1] + 1, g.G[2] + 1, gp[0], gp[1], gp[2], nrm);
        const float m2 = length2f(nrm[0], nrm[1], nrm[2]);
        float out = (D == 0 ? u : (D == 1 ? v : w))[f];
        if(m2 > FLT_MIN) {
            const float sq = sqrtf(m2);
            nrm[0] = nrm[0] / sq; nrm[1] = nrm[1] / sq; nrm[2] = nrm[2] / sq;
            const float dn = (vel[0] * nrm[0] + vel[1] * nrm[1]) + vel[2] * nrm[2];
            out = vel[D] - dn * nrm[D];
        }
        tmp[f] = out;
    }
}
template<int D>
__global__ void __launch_bounds__(256) k_constrain_apply(GridDesc g, const DevState* __restrict__ st,
                                                         const uint8_t* __restrict__ valid,
                                                         const float* __restrict__ weight,
                                                         const float* __restrict__ tmp, float* __restrict__ vel) {
    const int S[3] = {g.G[0] + (D == 0), g.G[1] + (D == 1), g.G[2] + (D == 2)};
    int lo[3], hi[3];
    if(!reach_box(st, kExtFull, S, lo, hi)) return;
    const long long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    for(long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nx * ny * nz;
        t += (long long)gridDim.x * blockDim.x) {
        const int i = lo[0] + (int)(t % nx), j = lo[1] + (int)((t / nx) % ny), k = lo[2] + (int)(t / (nx * ny));
        const size_t f = ((size_t)k * S[1] + j) * S[0] + i;
        if(valid[f] == 2 && weight[f] < FLT_MIN) vel[f] = tmp[f];
    }
}

// ----------------------------------------------------------------------------------
// G2P
// ----------------------------------------------------------------------------------
// FLIP_Solver::mapGrid2Particles (FLIP_Solver.cpp:99-111): v = lerp(v_grid, v_p + dv_grid,
// PIC_FLIP_ratio); APIC takes v_grid and C = grad v (APIC_Solver.cpp:95-117); AFLIP blends
// both (AFLIP_Solver.cpp:94-132).  kind: 0 FLIP, 1 APIC, 2 AFLIP.
template<bool DIFF>
__device__ __forceinline__ void grad_value_t(const float* __restrict__ a, const float* __restrict__ o, int sx, int sy,
                                             int sz, float px, float py, float pz, float cellSize, float out[3]) {
    // ArrayHelpers::interpolateGradientValue 3D (ArrayHelpers.cpp:275-302)
    int i, j, k;
    float fi, fj, fk;
    bary(px, i, fi, sx);
    bary(py, j, fj, sy);
    bary(pz, k, fk, sz);
    // 32-bit tap index (as interp_face)
    const unsigned usx = (unsigned)sx, sxy = usx * (unsigned)sy;
    const unsigned b = (unsigned)k * sxy + (unsigned)j * usx + (unsigned)i;
    const unsigned offs[8] = {0u, sxy, usx, sxy + usx, 1u, sxy + 1u, usx + 1u, sxy + usx + 1u};
    float vv[8]; // v000, v001, v010, v011, v100, v101, v110, v111
#pragma unroll
    for(int q = 0; q < 8; ++q) vv[q] = DIFF ? a[b + offs[q]] - o[b + offs[q]] : a[b + offs[q]];
    const float one = 1.0f;
    const float wx[8] = {-(one - fj) * (one - fk), -(one - fj) * fk, -fj * (one - fk), -fj * fk,
                         (one - fj) * (one - fk), (one - fj) * fk, fj * (one - fk), fj * fk};
    const float wy[8] = {-(one - fi) * (one - fk), -(one - fi) * fk, (one - fi) * (one - fk), (one - fi) * fk,
                         -fi * (one - fk), -fi * fk, fi * (one - fk), fi * fk};
    const float wz[8] = {-(one - fi) * (one - fj), (one - fi) * (one - fj), -(one - fi) * fj, (one - fi) * fj,
                         -fi * (one - fj), fi * (one - fj), -fi * fj, fi * fj};
    float s0 = vv[0] * wx[0], s1 = vv[0] * wy[0], s2 = vv[0] * wz[0];
#pragma unroll
    for(int q = 1; q < 8; ++q) { s0 = s0 + vv[q] * wx[q]; s1 = s1 + vv[q] * wy[q]; s2 = s2 + vv[q] * wz[q]; }
    out[0] = s0 / cellSize; out[1] = s1 / cellSize; out[2] = s2 / cellSize;
}
__device__ __forceinline__ void grad_value(const float* a, int sx, int sy, int sz, float px, float py, float pz,
                                           float cellSize, float out[3]) {
    grad_value_t<false>(a, nullptr, sx, sy, sz, px, py, pz, cellSize, out);
}
__device__ __forceinline__ void grad_value_diff(const float* a, const float* o, int sx, int sy, int sz, float px,
                                                float py, float pz, float cellSize, float out[3]) {
    grad_value_t<true>(a, o, sx, sy, sz, px, py, pz, cellSize, out);
}

__global__ void __launch_bounds__(256) k_g2p(int n, GridDesc g, const float* __restrict__ pos6, float* __restrict__ vel3,
                                             size_t stride, const float* __restrict__ u, const float* __restrict__ v,
                                             const float* __restrict__ w, const float* __restrict__ ou,
                                             const float* __restrict__ ov, const float* __restrict__ ow, float ratio,
                                             int kind, float* __restrict__ C9) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const float gx = (pos6[p] - g.bmin[0]) / g.dx;
    const float gy = (pos6[stride + p] - g.bmin[1]) / g.dx;
    const float gz = (pos6[2 * stride + p] - g.bmin[2]) / g.dx;
    const int G0 = g.G[0], G1 = g.G[1], G2 = g.G[2];
    float gv[3];
    if(kind == 1) {
        vel_from_grid(g, u, v, w, gx, gy, gz, gv);
#pragma unroll
        for(int d = 0; d < 3; ++d) vel3[d * stride + p] = gv[d];
    } else {
        // the grid velocity and its change at the particle, from the same taps
        float dg[3];
        interp_face_pair(u, ou, G0 + 1, G1, G2, gx, gy - 0.5f, gz - 0.5f, &gv[0], &dg[0]);
        interp_face_pair(v, ov, G0, G1 + 1, G2, gx - 0.5f, gy, gz - 0.5f, &gv[1], &dg[1]);
        interp_face_pair(w, ow, G0, G1, G2 + 1, gx - 0.5f, gy - 0.5f, gz, &gv[2], &dg[2]);
#pragma unroll
        for(int d = 0; d < 3; ++d) {
            const float pv = vel3[d * stride + p];
            vel3[d * stride + p] = (1.0f - ratio) * gv[d] + ratio * (pv + dg[d]);
        }
    }
    if(kind == 1 || kind == 2) {
        const float* arrs[3] = {u, v, w};
        const float* olds[3] = {ou, ov, ow};
        const int dims[3][3] = {{G0 + 1, G1, G2}, {G0, G1 + 1, G2}, {G0, G1, G2 + 1}};
        for(int d = 0; d < 3; ++d) {
            const float ptx = d == 0 ? gx : gx - 0.5f, pty = d == 1 ? gy : gy - 0.5f, ptz = d == 2 ? gz : gz - 0.5f;
            float gc[3];
            grad_value(arrs[d], dims[d][0], dims[d][1], dims[d][2], ptx, pty, ptz, g.dx, gc);
            if(kind == 1) {
#pragma unroll
                for(int c = 0; c < 3; ++c) C9[(size_t)(d * 3 + c) * stride + p] = gc[c];
            } else {
                // dGridC = interpolateGradientValue of dVels = velocities - oldVels
                // (AFLIP_Solver.cpp:121-130), differences formed tap by tap
                float dc[3];
                grad_value_diff(arrs[d], olds[d], dims[d][0], dims[d][1], dims[d][2], ptx, pty, ptz, g.dx, dc);
#pragma unroll
                for(int c = 0; c < 3; ++c) {
                    const size_t o_ = (size_t)(d * 3 + c) * stride + p;
                    C9[o_] = (1.0f - ratio) * gc[c] + ratio * (C9[o_] + dc[c]);
                }
            }
        }
    }
}

// ----------------------------------------------------------------------------------
// FLIP grid-to-particle transfer fused with the next sub-step's particle move
// ----------------------------------------------------------------------------------
// The next sub-step's size (PIC_Solver::advanceFrame, PIC_Solver.cpp:280-290, with
// timestepCFL, :342-349) from max|u| of the final grid of this sub-step, in the float
// operations the host uses (timestep_cfl in capi.cu): every thread forms the same value.
__device__ __forceinline__ float next_substep(unsigned maxvelBits, const NextStep& ns, float dx) {
    float ft = ns.frameTime;
    if(ft >= ns.frameDuration) ft = 0.f;  // a new frame starts
    const float m = __uint_as_float(maxvelBits);
    float maxVel = FLT_MIN;
    maxVel = (maxVel < m) ? m : maxVel;
    float ts = maxVel > FLT_MIN ? ns.cfl * (dx / maxVel) : FLT_MAX;
    if(ts < ns.minDt) ts = ns.minDt;
    else if(ts > ns.maxDt) ts = ns.maxDt;
    const float remaining = ns.frameDuration - ft;
    if(ft + ts >= ns.frameDuration) ts = remaining;
    else if(ft + 1.5f * ts >= ns.frameDuration) ts = remaining * 0.5f;
    return ts;
}

// FLIP_Solver::mapGrid2Particles (FLIP_Solver.cpp:99-111; KIND 0), APIC_Solver's and
// AFLIP_Solver's (the velocity and affine matrix of k_g2p; KIND 1, 2), then the next
// sub-step's PIC_Solver::moveParticles (PIC_Solver.cpp:353-373) and the first half of its
// counting sort: both read the same grid (the next sub-step starts from this one's
// velocities), and the move's first RK2 stage is the grid velocity the transfer has just
// interpolated at the particle.  The particle keeps its position of this sub-step (what
// callers read between sub-steps); the moved position goes to `moved`, and the next
// sub-step's sort gathers from there.  Identical arithmetic to k_g2p followed by k_advect.
template <int KIND>
__device__ __forceinline__ void g2p_move_body(Blk blk, int n, const GridDesc& g, float* __restrict__ p6, size_t stride,
                                              const float* __restrict__ u, const float* __restrict__ v,
                                              const float* __restrict__ w, const float* __restrict__ ou,
                                              const float* __restrict__ ov, const float* __restrict__ ow, float ratio,
                                              const NextStep& ns, float* __restrict__ moved,
                                              uint32_t* __restrict__ cellOf, uint32_t* __restrict__ slot,
                                              uint32_t* __restrict__ count, DevState* st,
                                              int* __restrict__ bboxPart, float* __restrict__ C9) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    const float substep = next_substep(st->maxvel_bits, ns, g.dx);
    const float sub = substep / (float)ns.advSteps;
    if(blk.x == 0 && threadIdx.x == 0) st->next_dt = substep;
    const int p = blk.x * blockDim.x + threadIdx.x;
    uint32_t c = 0xffffffffu;
    if(p < n) {
        float x = p6[p], y = p6[stride + p], z = p6[2 * stride + p];
        float gx = (x - g.bmin[0]) / g.dx, gy = (y - g.bmin[1]) / g.dx, gz = (z - g.bmin[2]) / g.dx;
        float gv[3];
        if(KIND == 1) {
            vel_from_grid(g, u, v, w, gx, gy, gz, gv);
#pragma unroll
            for(int d = 0; d < 3; ++d) p6[(3 + d) * stride + p] = gv[d];
        } else {
            // the grid velocity (getVelocityFromGrid) and its change (FLIP_Solver.cpp:125-133)
            // at the particle, from the same taps
            const int G0 = g.G[0], G1 = g.G[1], G2 = g.G[2];
            float dg[3];
            interp_face_pair(u, ou, G0 + 1, G1, G2, gx, gy - 0.5f, gz - 0.5f, &gv[0], &dg[0]);
            interp_face_pair(v, ov, G0, G1 + 1, G2, gx - 0.5f, gy, gz - 0.5f, &gv[1], &dg[1]);
            interp_face_pair(w, ow, G0, G1, G2 + 1, gx - 0.5f, gy - 0.5f, gz, &gv[2], &dg[2]);
            float* vel3 = p6 + 3 * stride;
#pragma unroll
            for(int d = 0; d < 3; ++d) {
                const float pv = vel3[d * stride + p];
                vel3[d * stride + p] = (1.0f - ratio) * gv[d] + ratio * (pv + dg[d]);
            }
        }
        if(KIND == 1 || KIND == 2) {
            // the affine matrix as k_g2p forms it
            const int G0 = g.G[0], G1 = g.G[1], G2 = g.G[2];
            const float* arrs[3] = {u, v, w};
            const float* olds[3] = {ou, ov, ow};
            const int dims[3][3] = {{G0 + 1, G1, G2}, {G0, G1 + 1, G2}, {G0, G1, G2 + 1}};
            for(int d = 0; d < 3; ++d) {
                const float ptx = d == 0 ? gx : gx - 0.5f, pty = d == 1 ? gy : gy - 0.5f, ptz = d == 2 ? gz : gz - 0.5f;
                float gc[3];
                grad_value(arrs[d], dims[d][0], dims[d][1], dims[d][2], ptx, pty, ptz, g.dx, gc);
                if(KIND == 1) {
#pragma unroll
                    for(int c = 0; c < 3; ++c) C9[(size_t)(d * 3 + c) * stride + p] = gc[c];
                } else {
                    float dc[3];
                    grad_value_diff(arrs[d], olds[d], dims[d][0], dims[d][1], dims[d][2], ptx, pty, ptz, g.dx, dc);
#pragma unroll
                    for(int c = 0; c < 3; ++c) {
                        const size_t o_ = (size_t)(d * 3 + c) * stride + p;
                        C9[o_] = (1.0f - ratio) * gc[c] + ratio * (C9[o_] + dc[c]);
                    }
                }
            }
        }
        for(int s = 0; s < ns.advSteps; ++s) {
            if(s > 0) {
                gx = (x - g.bmin[0]) / g.dx; gy = (y - g.bmin[1]) / g.dx; gz = (z - g.bmin[2]) / g.dx;
                vel_from_grid(g, u, v, w, gx, gy, gz, gv);
            }
            const float h = 0.5f * sub;
            const float mxp = x + h * gv[0], myp = y + h * gv[1], mzp = z + h * gv[2];
            gx = (mxp - g.bmin[0]) / g.dx; gy = (myp - g.bmin[1]) / g.dx; gz = (mzp - g.bmin[2]) / g.dx;
            float gm[3];
            vel_from_grid(g, u, v, w, gx, gy, gz, gm);
            x = x + sub * gm[0];
            y = y + sub * gm[1];
            z = z + sub * gm[2];
            constrain_particle(g, x, y, z);
        }
        moved[p] = x; moved[stride + p] = y; moved[2 * stride + p] = z;
        bool outside;
        int cc[3];
        c = cell_linear(g, (x - g.bmin[0]) / g.dx, (y - g.bmin[1]) / g.dx, (z - g.bmin[2]) / g.dx, outside, cc);
        if(outside) atomicOr(&st->next_flags, BNN_FLAG_OUT_OF_GRID);
        cellOf[p] = c;
#pragma unroll
        for(int d = 0; d < 3; ++d) { mn[d] = cc[d]; mx[d] = cc[d]; }
    }
    histogram_slot(c, p, count, slot);
    bbox_block_partial(bboxPart, blk.x, mn, mx);
}
template <int KIND>
__global__ void __launch_bounds__(256, 4) k_g2p_move(int n, GridDesc g, float* __restrict__ p6, size_t stride,
                                                  const float* __restrict__ u, const float* __restrict__ v,
                                                  const float* __restrict__ w, const float* __restrict__ ou,
                                                  const float* __restrict__ ov, const float* __restrict__ ow,
                                                  float ratio, NextStep ns, float* __restrict__ moved,
                                                  uint32_t* __restrict__ cellOf, uint32_t* __restrict__ slot,
                                                  uint32_t* __restrict__ count, DevState* st,
                                                  int* __restrict__ bboxPart, float* __restrict__ C9) {
    g2p_move_body<KIND>(own_blk(), n, g, p6, stride, u, v, w, ou, ov, ow, ratio, ns, moved, cellOf, slot, count, st,
                        bboxPart, C9);
}

// Start of a sub-step whose move already ran: the move's flags and occupied-cell box stay
__global__ void k_step_reset_moved(DevState* st) {
    st->flags = st->next_flags;
    st->next_flags = 0u;
    st->zero_phi = 0u;
    st->maxvel_bits = 0u;
}

// ----------------------------------------------------------------------------------
// Particle I/O
// ----------------------------------------------------------------------------------
__global__ void k_aos_to_soa(int n, const float* __restrict__ pos, const float* __restrict__ vel,
                             float* __restrict__ soa6, uint32_t* __restrict__ ids, size_t stride) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        soa6[d * stride + p] = pos[3 * (size_t)p + d];
        soa6[(3 + d) * stride + p] = vel[3 * (size_t)p + d];
    }
    ids[p] = (uint32_t)p;
}

// back to AoS in the caller's original order
__global__ void k_soa_to_aos(int n, const float* __restrict__ soa6, const uint32_t* __restrict__ ids,
                             float* __restrict__ pos, float* __restrict__ vel, size_t stride) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const uint32_t id = ids[p];
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        pos[3 * (size_t)id + d] = soa6[d * stride + p];
        vel[3 * (size_t)id + d] = soa6[(3 + d) * stride + p];
    }
}

// One AoS vec3 array to / from three SoA planes (ids: written as 0..n-1 on the way in,
// the caller's order on the way out)
__global__ void k_aos3_to_soa(int n, const float* __restrict__ aos, float* __restrict__ soa3,
                              uint32_t* __restrict__ ids, size_t stride) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
#pragma unroll
    for(int d = 0; d < 3; ++d) soa3[d * stride + p] = aos[3 * (size_t)p + d];
    if(ids) ids[p] = (uint32_t)p;
}

// planes of per-particle values from the current (sorted) order to the caller's order
__global__ void k_scatter_planes(int n, int planes, const float* __restrict__ src, const uint32_t* __restrict__ ids,
                                 float* __restrict__ dst, size_t stride) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const uint32_t id = ids[p];
    for(int k = 0; k < planes; ++k) dst[k * stride + id] = src[k * stride + p];
}

__global__ void k_soa3_to_aos(int n, const float* __restrict__ soa3, const uint32_t* __restrict__ ids,
                              float* __restrict__ aos, size_t stride) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const uint32_t id = ids[p];
#pragma unroll
    for(int d = 0; d < 3; ++d) aos[3 * (size_t)id + d] = soa3[d * stride + p];
}

// pressure scattered onto cells for BNN_FIELD_PRESSURE / BNN_FIELD_ACTIVE
__global__ void k_cells_from_rows(size_t nc, const float* __restrict__ phi, const uint32_t* __restrict__ aidx,
                                  const float* __restrict__ pr, float* __restrict__ out, int activeField) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= nc) return;
    if(activeField) out[c] = phi[c] < 0.f ? (float)(aidx[c] + 1) : 0.f;
    else out[c] = phi[c] < 0.f ? pr[aidx[c]] : 0.f;
}

__global__ void k_add_scalar(float* __restrict__ a, size_t n, float v) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) a[i] = a[i] + v;
}

__global__ void k_step_reset(DevState* st) {
    st->flags = 0u;
    st->next_flags = 0u;
    st->zero_phi = 0u;
    st->maxvel_bits = 0u;
    for(int d = 0; d < 3; ++d) { st->bbox[d] = INT_MAX; st->bbox[3 + d] = INT_MIN; }
}


// ----------------------------------------------------------------------------------
// Batched stages: one launch over all scenes of a batch (batch_step.cu).  Each block finds
// its scene and its block within the scene's share of the launch (seg_blk over the
// per-scene block prefix P) and runs the lone kernel's body there, on that scene's arrays.
// ----------------------------------------------------------------------------------
__global__ void kb_step_reset(const BScene* __restrict__ S, int ns) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if(q >= ns) return;
    DevState* st = S[q].dst;
    st->flags = S[q].moved ? st->next_flags : 0u;
    st->next_flags = 0u;
    st->zero_phi = 0u;
    st->maxvel_bits = 0u;
    st->nlarge = 0u;
    if(!S[q].moved)
        for(int d = 0; d < 3; ++d) { st->bbox[d] = INT_MAX; st->bbox[3 + d] = INT_MIN; }
}
__global__ void __launch_bounds__(256, 3) kb_advect(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)(c.n + 255) / 256, [&](Blk v) {
        advect_body(v, c.n, c.p6cur, c.p6cur + c.cap, c.p6cur + 2 * c.cap, c.U[0], c.U[1], c.U[2], c.g, c.sub,
                    c.advSteps, c.cellOf, c.slot, c.count, c.dst, c.bboxPart);
    });
}
// one block per scene: the occupied-cell box from the advection's per-block boxes
__global__ void __launch_bounds__(256) kb_bbox_final(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    bbox_final_body(b, (c.n + 255) / 256, c.bboxPart, c.dst);
}
__global__ void kb_scatter_index(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)(c.n + 255) / 256,
                   [&](Blk v) { scatter_index_body(v, c.n, c.cellOf, c.slot, c.cellStart, c.idcur, c.order, c.key); });
}
__global__ void __launch_bounds__(256, 4) kb_sort_buckets(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)((c.C + 255) / 256),
                   [&](Blk v) { sort_buckets_body(v, (int)c.C, c.cellStart, c.order, c.key, c.count, c.slot, c.dst); });
}
__global__ void __launch_bounds__(256) kb_sort_large(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    sort_large_body(b, c.cellStart, c.order, c.idcur, c.cellOf, c.slot, c.dst);
}
__global__ void kb_gather_particles(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)(c.n + 255) / 256, [&](Blk v) {
        gather_particles_body(v, c.n, c.order, c.p6cur, c.moved ? c.movedPos : c.p6cur, c.p6nxt, c.idcur, c.idnxt,
                              nullptr, nullptr, c.rec, c.g, c.cap);
    });
}
// Before the last layer after P2G: the FLIP backup starts at 0 and v at 0 - g dt (the
// values every face beyond the layer's region keeps; launch_extrapolate mode 1)
__global__ void kb_fill_backup(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    for(int d = 0; d < 3; ++d) {
        const size_t nf = (size_t)face_sx(c.g, d) * face_sy(c.g, d) * face_sz(c.g, d);
        fill_body(b, c.O[d], nf, 0.f);
        if(d == 1 && c.gdt != 0.f) fill_body(b, c.U[1], nf, 0.f - c.gdt);
    }
}
// Before the pressure update: its output arrays start at 0 / invalid
__global__ void kb_fill_update(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    for(int d = 0; d < 3; ++d) {
        const size_t nf = (size_t)face_sx(c.g, d) * face_sy(c.g, d) * face_sz(c.g, d);
        fill_body(b, c.B[d], nf, 0.f);
        for(size_t i = (size_t)b.x * blockDim.x + threadIdx.x; i < nf; i += (size_t)b.n * blockDim.x) c.VB[d][i] = 0;
    }
}
// Extrapolation layer `layer` of pass 1 (after P2G: U -> B -> U ..., backup and gravity on
// the last layer) or pass 2 (after the pressure update: B -> U -> B ..., the CFL maximum on
// the last layer), as launch_extrapolate builds them
__global__ void __launch_bounds__(256, 4) kb_extrapolate(const BScene* __restrict__ S, const unsigned* __restrict__ P,
                                                         int ns, int pass, int layer) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    ExtLayer a;
    const bool even = layer % 2 == 0;
    a.mode = layer == 3 ? pass : 0;
    for(int d = 0; d < 3; ++d) {
        a.S[d][0] = face_sx(c.g, d); a.S[d][1] = face_sy(c.g, d); a.S[d][2] = face_sz(c.g, d);
        float* A = pass == 1 ? c.U[d] : c.B[d];
        uint8_t* VA_ = pass == 1 ? c.VA[d] : c.VB[d];
        float* Bv = pass == 1 ? c.B[d] : c.U[d];
        uint8_t* VB_ = pass == 1 ? c.VB[d] : c.VA[d];
        a.gin[d] = even ? A : Bv;
        a.vin[d] = even ? VA_ : VB_;
        a.gout[d] = even ? Bv : A;
        a.vout[d] = even ? VB_ : VA_;
        a.oldOut[d] = pass == 1 ? c.O[d] : nullptr;
        a.gdt[d] = (a.mode == 1 && d == 1) ? c.gdt : 0.f;
    }
    extrapolate3_body(b, a, c.dst);
}
__global__ void kb_active_flags(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)((c.C + 255) / 256), [&](Blk v) { active_flags_body(v, c.g, c.phi, c.flag, c.dst); });
}
__global__ void kb_active_rows(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)((c.C + 255) / 256), [&](Blk v) { active_rows_body(v, c.C, c.flag, c.aidx, c.rowCell); });
}
__global__ void kb_build_rows(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    virtual_blocks(b, (unsigned)(c.nrows + 255) / 256, [&](Blk v) {
        build_rows_body<false>(v, c.g, c.nrows, c.rowCell, c.phi, c.aidx, c.U[0], c.U[1], c.U[2], nullptr, nullptr,
                               nullptr, c.substep, c.rhs, c.diag, c.invd, c.nbr, nullptr, c.dst);
    });
}
template<int D>
__global__ void __launch_bounds__(256) kb_update_velocity(const BScene* __restrict__ S, const unsigned* __restrict__ P,
                                                          int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    update_velocity_body<D>(b, c.g, c.dst, c.phi, c.aidx, c.pressure, c.substep, c.U[D], c.B[D], c.VB[D], nullptr);
}
// one thread per scene: the occupied-cell box of the fused move starts empty
__global__ void kb_bbox_reset(const BScene* __restrict__ S, int ns) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if(q >= ns) return;
    DevState* st = S[q].dst;
    for(int d = 0; d < 3; ++d) { st->bbox[d] = INT_MAX; st->bbox[3 + d] = INT_MIN; }
}
// the fused grid-to-particle transfer + next move, on the final velocities of this
// sub-step (the pass-2 extrapolation leaves them in B)
__global__ void __launch_bounds__(256, 3) kb_g2p_move(const BScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const BScene& c = S[q];
    g2p_move_body<0>(b, c.n, c.g, c.p6nxt, c.cap, c.B[0], c.B[1], c.B[2], c.O[0], c.O[1], c.O[2], c.ratio, c.ns,
                     c.movedPos, c.cellOf, c.slot, c.count, c.dst, c.bboxPart, nullptr);
}
// one thread per scene: its pressure rows (the active-cell numbering's total)
__global__ void kb_gather_rows(const BScene* __restrict__ S, int ns, unsigned* __restrict__ out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if(q < ns) out[q] = S[q].aidx[S[q].C];
}
__global__ void kb_gather_state(const BScene* __restrict__ S, int ns, DevState* __restrict__ out) {
    const int q = blockIdx.x;
    if(q >= ns) return;
    const unsigned* src = (const unsigned*)S[q].dst;
    unsigned* dst = (unsigned*)(out + q);
    for(int i = threadIdx.x; i < (int)(sizeof(DevState) / 4); i += blockDim.x) dst[i] = src[i];
}

// ----------------------------------------------------------------------------------
// Launchers
// ----------------------------------------------------------------------------------
static inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

void launch_advect(int n, float* p6, size_t stride, const float* const* U, const GridDesc& g, float sub, int steps,
                   uint32_t* cellOf, uint32_t* slot, uint32_t* count, DevState* st, int* bboxPart, cudaStream_t s) {
    if(n == 0) return;
    const unsigned blocks = nblk(n);
    { k_advect<<<blocks, 256, 0, s>>>(n, p6, p6 + stride, p6 + 2 * stride, U[0], U[1], U[2], g, sub, steps, cellOf, slot,
                                     count, st, bboxPart); bnn_note_launch(); }
    const unsigned fb = blocks < 148u * 4u * 256u ? (blocks + 255u) / 256u : 148u * 4u;
    { k_bbox_final<<<fb, 256, 0, s>>>((int)blocks, bboxPart, st); bnn_note_launch(); }
}
void launch_cell_histogram(int n, const float* p6, size_t stride, const GridDesc& g, uint32_t* cellOf, uint32_t* slot,
                           uint32_t* count, DevState* st, cudaStream_t s) {
    if(n == 0) return;
    { k_cell_histogram<<<nblk(n), 256, 0, s>>>(n, p6, p6 + stride, p6 + 2 * stride, g, cellOf, slot, count, st); bnn_note_launch(); }
}
// cellOf and slot are free once the index is scattered: slot lists the crowded buckets,
// cellOf holds their unsorted order while k_sort_large rewrites them
void launch_sort_finish(int n, size_t ncells, uint32_t* cellOf, uint32_t* slot, const uint32_t* cellStart,
                        uint32_t* order, uint32_t* key, uint32_t* count, const float* src6, const float* srcPos,
                        float* dst6, const uint32_t* idSrc, uint32_t* idDst, const float* cSrc, float* cDst,
                        float4* rec, const GridDesc& g, size_t stride, DevState* st, cudaStream_t s,
                        cudaEvent_t gatherAfter) {
    if(n > 0) { k_scatter_index<<<nblk(n), 256, 0, s>>>(n, cellOf, slot, cellStart, idSrc, order, key); bnn_note_launch(); }
    cudaMemsetAsync(&st->nlarge, 0, sizeof(unsigned), s);
    { k_sort_buckets<<<nblk(ncells), 256, 0, s>>>((int)ncells, cellStart, order, key, count, slot, st); bnn_note_launch(); }
    if(n > 16) { k_sort_large<<<8 * 148, 256, 0, s>>>(cellStart, order, idSrc, cellOf, slot, st); bnn_note_launch(); }
    // src6's velocity planes may still be arriving on another stream until this event
    if(gatherAfter) cudaStreamWaitEvent(s, gatherAfter, 0);
    if(n > 0)
        { k_gather_particles<<<nblk(n), 256, 0, s>>>(n, order, src6, srcPos ? srcPos : src6, dst6, idSrc, idDst, cSrc, cDst,
                                                    rec, g, stride); bnn_note_launch(); }
}
// PIC grid advection of all three components; U[d] / B[d] are swapped after each one
void launch_advect_grid(const GridDesc& g, float** U, float** B, float dt, cudaStream_t s) {
    const float inv = 1.0f / g.dx;
    for(int d = 0; d < 3; ++d) {
        const size_t nf = (size_t)face_sx(g, d) * face_sy(g, d) * face_sz(g, d);
        if(d == 0) { k_advect_grid<0><<<nblk(nf), 256, 0, s>>>(g, U[0], U[1], U[2], inv, dt, B[0]); bnn_note_launch(); }
        if(d == 1) { k_advect_grid<1><<<nblk(nf), 256, 0, s>>>(g, U[0], U[1], U[2], inv, dt, B[1]); bnn_note_launch(); }
        if(d == 2) { k_advect_grid<2><<<nblk(nf), 256, 0, s>>>(g, U[0], U[1], U[2], inv, dt, B[2]); bnn_note_launch(); }
        float* t = U[d];
        U[d] = B[d];
        B[d] = t;
    }
}

static constexpr unsigned kRegionBlocks = 148u * 8u;

void launch_correct_positions(int n, const GridDesc& g, const float* p6, size_t stride, const uint32_t* ids,
                              const uint32_t* cellStart, float radius2, float threshold2, float jitterScale,
                              float kSpring, int advSteps, unsigned long long step, float* out3, cudaStream_t s) {
    if(n == 0) return;
    { k_correct_positions<<<nblk(n), 256, 0, s>>>(n, g, p6, p6 + stride, p6 + 2 * stride, ids, cellStart, radius2,
                                                 threshold2, jitterScale, kSpring, advSteps, step, out3,
                                                 out3 + stride, out3 + 2 * stride); bnn_note_launch(); }
}
void launch_rebin(int n, const float* p6, size_t stride, const GridDesc& g, uint32_t* cellOf, uint32_t* slot,
                  uint32_t* count, DevState* st, cudaStream_t s) {
    { k_bbox_reset<<<1, 1, 0, s>>>(st); bnn_note_launch(); }
    if(n == 0) return;
    const unsigned blocks = nblk(n) < kRegionBlocks ? nblk(n) : kRegionBlocks;
    { k_rebin<<<blocks, 256, 0, s>>>(n, p6, p6 + stride, p6 + 2 * stride, g, cellOf, slot, count, st); bnn_note_launch(); }
}

void launch_maxabs(const float* a, size_t n, unsigned* maxBits, cudaStream_t s) {
    if(n) { k_maxabs<<<kRegionBlocks, 256, 0, s>>>(a, n, maxBits); bnn_note_launch(); }
}  // resident blocks of the region kernels

// 4 layers per component; A holds the input and receives the result (4 is even).  Mode 1
// first writes the values the last layer gives every face beyond its region: backup 0,
// and v = 0 - gravityDt (A holds 0 there).
void launch_extrapolate(const GridDesc& g, float* const* A, uint8_t* const* VA, float* const* B, uint8_t* const* VB,
                        int lastMode, float* const* oldOut, float gravityDt, DevState* st, cudaStream_t s) {
    for(int layer = 0; layer < 4; ++layer) {
        ExtLayer a;
        a.mode = layer == 3 ? lastMode : 0;
        for(int d = 0; d < 3; ++d) {
            a.S[d][0] = face_sx(g, d); a.S[d][1] = face_sy(g, d); a.S[d][2] = face_sz(g, d);
            const size_t nf = (size_t)a.S[d][0] * a.S[d][1] * a.S[d][2];
            a.gin[d] = (layer % 2 == 0) ? A[d] : B[d];
            a.vin[d] = (layer % 2 == 0) ? VA[d] : VB[d];
            a.gout[d] = (layer % 2 == 0) ? B[d] : A[d];
            a.vout[d] = (layer % 2 == 0) ? VB[d] : VA[d];
            a.oldOut[d] = oldOut ? oldOut[d] : nullptr;
            a.gdt[d] = (a.mode == 1 && d == 1) ? gravityDt : 0.f;
            if(a.mode == 1) {
                cudaMemsetAsync(oldOut[d], 0, nf * sizeof(float), s);
                if(a.gdt[d] != 0.f) { k_fill<<<kRegionBlocks, 256, 0, s>>>(a.gout[d], nf, 0.f - a.gdt[d]); bnn_note_launch(); }
            }
        }
        { k_extrapolate3<<<kRegionBlocks, 256, 0, s>>>(a, st); bnn_note_launch(); }
    }
}
void launch_active_flags(const GridDesc& g, const float* phi, uint32_t* flag, DevState* st, cudaStream_t s) {
    size_t nc = (size_t)g.G[0] * g.G[1] * g.G[2];
    { k_active_flags<<<nblk(nc), 256, 0, s>>>(g, phi, flag, st); bnn_note_launch(); }
}
void launch_active_rows(size_t nc, const uint32_t* flag, const uint32_t* idx, uint32_t* rowCell, cudaStream_t s) {
    { k_active_rows<<<nblk(nc), 256, 0, s>>>(nc, flag, idx, rowCell); bnn_note_launch(); }
}
// W (optional): face weights of u, v, w; with them the off-diagonal values go to coef
void launch_build_rows(const GridDesc& g, int nrows, const uint32_t* rowCell, const float* phi, const uint32_t* aidx,
                       const float* const* U, const float* const* W, float dt, float* rhs, float* diag, float* invdiag,
                       int32_t* nbr, float* coef, DevState* st, cudaStream_t s) {
    if(nrows == 0) return;
    if(W) {
        k_build_rows<true><<<nblk(nrows), 256, 0, s>>>(g, nrows, rowCell, phi, aidx, U[0], U[1], U[2], W[0], W[1], W[2],
                                                     dt, rhs, diag, invdiag, nbr, coef, st);
    } else {
        k_build_rows<false><<<nblk(nrows), 256, 0, s>>>(g, nrows, rowCell, phi, aidx, U[0], U[1], U[2], nullptr, nullptr,
                                                      nullptr, dt, rhs, diag, invdiag, nbr, nullptr, st);
    }
    bnn_note_launch();
}
// Reads velIn, writes the projected faces to velOut / validOut (zeroed here first).
void launch_update_velocity(const GridDesc& g, const DevState* st, const float* phi, const uint32_t* aidx,
                            const float* pressure, float dt, float* const* velIn, float* const* velOut,
                            uint8_t* const* validOut, const float* const* W, cudaStream_t s) {
    for(int d = 0; d < 3; ++d) {
        const size_t nf = (size_t)face_sx(g, d) * face_sy(g, d) * face_sz(g, d);
        cudaMemsetAsync(velOut[d], 0, nf * sizeof(float), s);
        cudaMemsetAsync(validOut[d], 0, nf, s);
    }
    { k_update_velocity<0><<<kRegionBlocks, 256, 0, s>>>(g, st, phi, aidx, pressure, dt, velIn[0], velOut[0], validOut[0], W ? W[0] : nullptr); bnn_note_launch(); }
    { k_update_velocity<1><<<kRegionBlocks, 256, 0, s>>>(g, st, phi, aidx, pressure, dt, velIn[1], velOut[1], validOut[1], W ? W[1] : nullptr); bnn_note_launch(); }
    { k_update_velocity<2><<<kRegionBlocks, 256, 0, s>>>(g, st, phi, aidx, pressure, dt, velIn[2], velOut[2], validOut[2], W ? W[2] : nullptr); bnn_note_launch(); }
}
// Node SDF of the boundary objects and the face weights it gives
void launch_boundary_grid(const GridDesc& g, float* nodeSdf, float* const* W, cudaStream_t s) {
    { k_node_sdf<<<kRegionBlocks, 256, 0, s>>>(g, nodeSdf); bnn_note_launch(); }
    { k_face_weights<0><<<kRegionBlocks, 256, 0, s>>>(g, nodeSdf, W[0]); bnn_note_launch(); }
    { k_face_weights<1><<<kRegionBlocks, 256, 0, s>>>(g, nodeSdf, W[1]); bnn_note_launch(); }
    { k_face_weights<2><<<kRegionBlocks, 256, 0, s>>>(g, nodeSdf, W[2]); bnn_note_launch(); }
}
void launch_solid_extend(const GridDesc& g, const float* nodeSdf, float* phi, cudaStream_t s) {
    { k_solid_extend<<<kRegionBlocks, 256, 0, s>>>(g, nodeSdf, phi); bnn_note_launch(); }
}
// constrainGridVelocity over U (components in order, each reading the ones before it as
// already constrained); T is scratch of the face arrays' sizes
void launch_constrain_velocity(const GridDesc& g, const DevState* st, float* const* U, uint8_t* const* V,
                               float* const* W, const float* nodeSdf, float* const* T, cudaStream_t s) {
    { k_constrain_compute<0><<<kRegionBlocks, 256, 0, s>>>(g, st, U[0], U[1], U[2], V[0], W[0], nodeSdf, T[0]); bnn_note_launch(); }
    { k_constrain_apply<0><<<kRegionBlocks, 256, 0, s>>>(g, st, V[0], W[0], T[0], U[0]); bnn_note_launch(); }
    { k_constrain_compute<1><<<kRegionBlocks, 256, 0, s>>>(g, st, U[0], U[1], U[2], V[1], W[1], nodeSdf, T[1]); bnn_note_launch(); }
    { k_constrain_apply<1><<<kRegionBlocks, 256, 0, s>>>(g, st, V[1], W[1], T[1], U[1]); bnn_note_launch(); }
    { k_constrain_compute<2><<<kRegionBlocks, 256, 0, s>>>(g, st, U[0], U[1], U[2], V[2], W[2], nodeSdf, T[2]); bnn_note_launch(); }
    { k_constrain_apply<2><<<kRegionBlocks, 256, 0, s>>>(g, st, V[2], W[2], T[2], U[2]); bnn_note_launch(); }
}
void launch_g2p(int n, const GridDesc& g, float* p6, size_t stride, const float* const* U, const float* const* O,
                float ratio, int kind, float* C9, cudaStream_t s) {
    if(n == 0) return;
    { k_g2p<<<nblk(n), 256, 0, s>>>(n, g, p6, p6 + 3 * stride, stride, U[0], U[1], U[2], O[0], O[1], O[2], ratio, kind,
                                  C9); bnn_note_launch(); }
}
void launch_aos_to_soa(int n, const float* pos, const float* vel, float* soa6, uint32_t* ids, size_t stride,
                       cudaStream_t s) {
    if(n == 0) return;
    { k_aos_to_soa<<<nblk(n), 256, 0, s>>>(n, pos, vel, soa6, ids, stride); bnn_note_launch(); }
}
void launch_soa_to_aos(int n, const float* soa6, const uint32_t* ids, float* pos, float* vel, size_t stride,
                       cudaStream_t s) {
    if(n == 0) return;
    { k_soa_to_aos<<<nblk(n), 256, 0, s>>>(n, soa6, ids, pos, vel, stride); bnn_note_launch(); }
}
void launch_aos3_to_soa(int n, const float* aos, float* soa3, uint32_t* ids, size_t stride, cudaStream_t s) {
    if(n == 0) return;
    { k_aos3_to_soa<<<nblk(n), 256, 0, s>>>(n, aos, soa3, ids, stride); bnn_note_launch(); }
}
void launch_scatter_planes(int n, int planes, const float* src, const uint32_t* ids, float* dst, size_t stride,
                           cudaStream_t s) {
    if(n == 0) return;
    { k_scatter_planes<<<nblk(n), 256, 0, s>>>(n, planes, src, ids, dst, stride); bnn_note_launch(); }
}
void launch_soa3_to_aos(int n, const float* soa3, const uint32_t* ids, float* aos, size_t stride, cudaStream_t s) {
    if(n == 0) return;
    { k_soa3_to_aos<<<nblk(n), 256, 0, s>>>(n, soa3, ids, aos, stride); bnn_note_launch(); }
}
void launch_add_scalar(float* a, size_t n, float v, cudaStream_t s) { { k_add_scalar<<<nblk(n), 256, 0, s>>>(a, n, v); bnn_note_launch(); } }
void launch_step_reset(DevState* st, cudaStream_t s) { { k_step_reset<<<1, 1, 0, s>>>(st); bnn_note_launch(); } }
void launch_step_reset_moved(DevState* st, cudaStream_t s) { { k_step_reset_moved<<<1, 1, 0, s>>>(st); bnn_note_launch(); } }
// FLIP grid-to-particle transfer + the next sub-step's move; the occupied-cell box is
// rebuilt for the next sub-step
void launch_g2p_move(int n, const GridDesc& g, float* p6, size_t stride, const float* const* U, const float* const* O,
                     float ratio, int kind, float* C9, const NextStep& ns, float* moved, uint32_t* cellOf,
                     uint32_t* slot, uint32_t* count, DevState* st, int* bboxPart, cudaStream_t s) {
    { k_bbox_reset<<<1, 1, 0, s>>>(st); bnn_note_launch(); }
    if(n == 0) return;
    const unsigned blocks = nblk(n);
    auto k = kind == 1 ? k_g2p_move<1> : kind == 2 ? k_g2p_move<2> : k_g2p_move<0>;
    { k<<<blocks, 256, 0, s>>>(n, g, p6, stride, U[0], U[1], U[2], O[0], O[1], O[2], ratio, ns, moved, cellOf, slot,
                               count, st, bboxPart, C9); bnn_note_launch(); }
    const unsigned fb = blocks < 148u * 4u * 256u ? (blocks + 255u) / 256u : 148u * 4u;
    { k_bbox_final<<<fb, 256, 0, s>>>((int)blocks, bboxPart, st); bnn_note_launch(); }
}
// Batched stages (kernels above): `blocks` = P[ns], the launch's total
void launch_batch_stage(BatchStage stage, const BScene* S, const unsigned* P, int ns, unsigned blocks, cudaStream_t s,
                        int pass, int layer) {
    if(ns == 0) return;
    const unsigned per = (unsigned)((ns + 127) / 128);
    switch(stage) {
    case BatchStage::StepReset: kb_step_reset<<<per, 128, 0, s>>>(S, ns); break;
    case BatchStage::BboxReset: kb_bbox_reset<<<per, 128, 0, s>>>(S, ns); break;
    default:
        if(blocks == 0) return;
        switch(stage) {
        case BatchStage::Advect: kb_advect<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::BboxFinal: kb_bbox_final<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::ScatterIndex: kb_scatter_index<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::SortBuckets: kb_sort_buckets<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::SortLarge: kb_sort_large<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::Gather: kb_gather_particles<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::FillBackup: kb_fill_backup<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::FillUpdate: kb_fill_update<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::Extrapolate: kb_extrapolate<<<blocks, 256, 0, s>>>(S, P, ns, pass, layer); break;
        case BatchStage::ActiveFlags: kb_active_flags<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::ActiveRows: kb_active_rows<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::BuildRows: kb_build_rows<<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::UpdateU: kb_update_velocity<0><<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::UpdateV: kb_update_velocity<1><<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::UpdateW: kb_update_velocity<2><<<blocks, 256, 0, s>>>(S, P, ns); break;
        case BatchStage::G2PMove: kb_g2p_move<<<blocks, 256, 0, s>>>(S, P, ns); break;
        default: return;
        }
    }
    bnn_note_launch();
}
void launch_batch_gather_rows(const BScene* S, int ns, unsigned* out, cudaStream_t s) {
    if(ns) { kb_gather_rows<<<(ns + 127) / 128, 128, 0, s>>>(S, ns, out); bnn_note_launch(); }
}
void launch_batch_gather_state(const BScene* S, int ns, DevState* out, cudaStream_t s) {
    if(ns) { kb_gather_state<<<ns, 128, 0, s>>>(S, ns, out); bnn_note_launch(); }
}

void launch_cells_from_rows(size_t nc, const float* phi, const uint32_t* aidx, const float* pr, float* out, int active,
                            cudaStream_t s) {
    { k_cells_from_rows<<<nblk(nc), 256, 0, s>>>(nc, phi, aidx, pr, out, active); bnn_note_launch(); }
}

} // namespace bnn
