// P2G (non-affine FLIP) and the fluid SDF in one tiled pass over the cell-sorted particles.
//
// FLIP_Solver::mapParticles2Grid (FLIP_Solver.cpp:57-95) splats every particle onto the 8
// faces of its trilinear stencil per component with CAS float atomics, so the reference
// has no fixed summation order.  Here each face's sums are formed in one fixed two-level
// order, independent of the launch shape:
//   1. per cell and per face the cell's particles can reach, a partial sum over the cell's
//      particles in id order (particles are sorted by (cell, id));
//   2. per face, the partials of its candidate cells added in (y, z, x)-major cell order:
//      two cells along the component's own axis, three along the others.
// Both sums start at +0.  The products are the reference's: weight = wx * wy * wz left to
// right (ArrayHelpers::getCoordinatesAndWeights, ArrayHelpers.cpp:50-76), momentum =
// weight * v.  The oracle's canonical mode (mapP2GCanonical) sums in the same order.
//
// The fluid SDF (PIC_Solver::computeFluidSDF, PIC_Solver.cpp:601-652) rides along: per cell
// the minimum squared distance of its particles to each of the 27 neighbouring cell
// centres, then per cell the minimum over its 27 neighbours' partials.  min is exact, so
// this equals the reference's locked scatter bit for bit; sqrtf (correctly rounded) and the
// radius subtraction are non-decreasing, so one square root per cell gives the minimum of
// the per-particle distances.
//
// Work layout.  A block owns a tile of kTX x kTZ face columns (x, z) and walks kYC face
// layers along y, the gravity axis (Earth gravity is -y, ParticleSolverData.cpp:196-200):
// a liquid piles up in the cells above the floor, and walking y makes every such crowded
// layer one layer that all columns of every tile share, instead of a long serial walk
// inside the few tiles that hold the floor.  A block has one thread per cell of its tile
// and the tile's 1-cell halo (warps are rows of 32 cells along x: 30 interior columns and a
// halo cell each side).  For each cell layer it needs, every thread forms its cell's
// partials into shared memory, one component at a time, then the interior threads add the
// partials their faces need to register accumulators for the three face layers the cell
// layer reaches.  Each particle record is therefore read once per block (plus the halo)
// instead of once per candidate face, the weight of a particle is formed once per reached
// slot, and no thread forms two cells' partials while the rest of the block waits.
//
// Input: one 16-byte record per particle and component, written by the sort's gather
// (flip_kernels.cu, k_gather_particles): plane D < 3 holds {e_x, e_y, e_z, v_D}, e_a the
// stencil fraction along axis a with the sign bit set when the stencil's base index is the
// particle's (sorted) cell - 1 instead of the cell itself; plane 3 holds the position.
#include "bnn_internal.cuh"

#include <atomic>
#include <cfloat>
#include <climits>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

namespace bnn {

namespace {
// A thread per cell of the tile plus its 1-cell halo: a warp is one row of 32 cells along x
// (30 interior columns and one halo cell each side), TZ + 2 rows along z.  Every thread
// forms the partials of exactly one cell, and the interior threads own the faces.  A block
// walks YC face layers along y.  The shape changes only which block forms which sums, not
// the sums: every shape gives the same bits, so the tuner (tile_tuner) may pick any.
constexpr int kHX = 32, kTX = kHX - 2;      // cells per row, interior face columns along x
constexpr int kPartials = 36;              // 18 face slots x (momentum, weight); the SDF has 27
template<int TZ, int YC>
struct Shape {
    static constexpr int kTZ = TZ;             // interior face columns along z
    static constexpr int kHZ = TZ + 2;
    static constexpr int kYC = YC;             // face layers per block along y (the walk)
    static constexpr int kNH = kHX * kHZ;      // cells of one layer whose partials the tile needs
    static constexpr int kThreads = kNH;
    static constexpr int kMinBlocks = 768 / kThreads > 0 ? 768 / kThreads : 1;
    static constexpr size_t kSmemBytes = sizeof(float) * kPartials * kNH;
};
// The shapes the tuner chooses from (index = bnn tile-shape id); 0 is the default
using S0 = Shape<6, 8>;
using S1 = Shape<4, 8>;
using S2 = Shape<6, 4>;
using S3 = Shape<4, 4>;
using S4 = Shape<6, 16>;
using S5 = Shape<8, 8>;

// Weights along one axis of a component's stencil, by face offset from the particle's
// cell.  The component's own axis: offsets {0, +1}, the base is always the cell.  Other
// axes: offsets {-1, 0, +1}; base cell - 1 (sign bit set) reaches offsets -1, 0, base cell
// reaches 0, +1.  Unreached offsets weigh exactly 0.
__device__ __forceinline__ void own_axis(float e, float w[2]) {
    w[0] = 1.0f - e;
    w[1] = e;
}
__device__ __forceinline__ void side_axis(float e, float w[3]) {
    const bool low = __float_as_int(e) < 0;
    const float f = fabsf(e);
    const float a = 1.0f - f;
    w[0] = low ? a : 0.0f;
    w[1] = low ? f : a;
    w[2] = low ? 0.0f : f;
}

struct TileArgs {
    GridDesc g;
    const DevState* st;
    const uint32_t* cellStart;
    const float4* rec;  // plane stride `stride`
    size_t stride;
    float* out[3];
    uint8_t* valid[3];
    float* phi;
    const float* C9;    // APIC / AFLIP: the sorted particles' affine matrices (9 planes, stride `stride`)
};

// Does the cell box [lo, hi] meet the occupied-cell box?
__device__ __forceinline__ bool meets_particles(const DevState* st, const int lo[3], const int hi[3]) {
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const int bl = st->bbox[d], bh = st->bbox[3 + d];
        if(bh < bl) return false;
        if(hi[d] < bl || lo[d] > bh) return false;
    }
    return true;
}

// The particles [b, e) of halo cell h of the current cell layer (none for a halo cell
// outside the grid), read once per layer for the four passes over them
__device__ __forceinline__ void cell_range(const TileArgs& a, int x0, int z0, int cy, int h, uint32_t& b, uint32_t& e) {
    const int cx = x0 - 1 + h % kHX, cz = z0 - 1 + h / kHX;
    b = e = 0u;
    if(cx >= 0 && cx < a.g.G[0] && cz >= 0 && cz < a.g.G[2]) {
        const size_t c = ((size_t)cz * a.g.G[1] + cy) * a.g.G[0] + cx;
        b = __ldg(a.cellStart + c);
        e = __ldg(a.cellStart + c + 1);
    }
}

// Partials of component D for halo cell h (particles [b, e)) into sm (slot-major planes).
// AFF (APIC / AFLIP, APIC_Solver.cpp:53-91): a particle's momentum at a face is
// weight * (v + C_D . (x_face - x_p)), x_face the face's world position
// (Grid::getWorldCoordinate, Grid.h:181-184), in the reference's association.
template<int D, class SH, bool AFF = false>
__device__ __forceinline__ void cell_partials(const TileArgs& a, int h, uint32_t b, uint32_t e, float* __restrict__ sm,
                                              int x0 = 0, int z0 = 0, int cy = 0) {
    constexpr int kNH = SH::kNH;
    constexpr int NX = D == 0 ? 2 : 3, NY = D == 1 ? 2 : 3, NZ = D == 2 ? 2 : 3;
    constexpr int NS = NX * NY * NZ;
    float S[NS], W[NS];
#pragma unroll
    for(int s = 0; s < NS; ++s) { S[s] = 0.0f; W[s] = 0.0f; }
    // AFF: world coordinates of the faces the slots address (slot i along axis a is the face
    // at offset i from the cell on the component's own axis, i - 1 on the others)
    float gpx[NX], gpy[NY], gpz[NZ];
    if constexpr(AFF) {
        const int cx = x0 - 1 + h % kHX, cz = z0 - 1 + h / kHX;
#pragma unroll
        for(int i = 0; i < NX; ++i) gpx[i] = ((float)(cx + (D == 0 ? i : i - 1)) + (D == 0 ? 0.f : 0.5f)) * a.g.dx + a.g.bmin[0];
#pragma unroll
        for(int i = 0; i < NY; ++i) gpy[i] = ((float)(cy + (D == 1 ? i : i - 1)) + (D == 1 ? 0.f : 0.5f)) * a.g.dx + a.g.bmin[1];
#pragma unroll
        for(int i = 0; i < NZ; ++i) gpz[i] = ((float)(cz + (D == 2 ? i : i - 1)) + (D == 2 ? 0.f : 0.5f)) * a.g.dx + a.g.bmin[2];
    }
    {
        const float4* __restrict__ recD = a.rec + (size_t)D * a.stride;
        // the next record is loaded while this one is summed
        float4 Ln = b < e ? __ldg(recD + b) : make_float4(0.f, 0.f, 0.f, 0.f);
        for(uint32_t q = b; q < e; ++q) {
            const float4 L = Ln;
            if(q + 1 < e) Ln = __ldg(recD + q + 1);
            float wx[NX], wy[NY], wz[NZ];
            if constexpr(D == 0) own_axis(L.x, wx); else side_axis(L.x, wx);
            if constexpr(D == 1) own_axis(L.y, wy); else side_axis(L.y, wy);
            if constexpr(D == 2) own_axis(L.z, wz); else side_axis(L.z, wz);
            float c0 = 0.f, c1 = 0.f, c2 = 0.f, dxp[NX], dyp[NY], dzp[NZ];
            if constexpr(AFF) {
                const float4 P = __ldg(a.rec + 3 * a.stride + q);
                const float* __restrict__ Cd = a.C9 + (size_t)(3 * D) * a.stride;
                c0 = __ldg(Cd + q);
                c1 = __ldg(Cd + a.stride + q);
                c2 = __ldg(Cd + 2 * a.stride + q);
#pragma unroll
                for(int i = 0; i < NX; ++i) dxp[i] = gpx[i] - P.x;
#pragma unroll
                for(int i = 0; i < NY; ++i) dyp[i] = gpy[i] - P.y;
#pragma unroll
                for(int i = 0; i < NZ; ++i) dzp[i] = gpz[i] - P.z;
            }
#pragma unroll
            for(int ix = 0; ix < NX; ++ix)
#pragma unroll
                for(int iy = 0; iy < NY; ++iy) {
                    const float wxy = wx[ix] * wy[iy];
                    float cxy = 0.f;
                    if constexpr(AFF) cxy = c0 * dxp[ix] + c1 * dyp[iy];
#pragma unroll
                    for(int iz = 0; iz < NZ; ++iz) {
                        const int s = (ix * NY + iy) * NZ + iz;
                        const float w = wxy * wz[iz];
                        if constexpr(AFF) {
                            const float dotv = cxy + c2 * dzp[iz];
                            S[s] = S[s] + w * (L.w + dotv);
                        } else {
                            S[s] = S[s] + w * L.w;
                        }
                        W[s] = W[s] + w;
                    }
                }
        }
    }
#pragma unroll
    for(int s = 0; s < NS; ++s) {
        sm[(2 * s) * kNH + h] = S[s];
        sm[(2 * s + 1) * kNH + h] = W[s];
    }
}

// The face (x0 + tx, z0 + tz) of component D adds the partials of its candidate cells of
// this layer, cells in ascending (z, x) order, into its accumulators for face layers
// cy - 1 + j.
template<int D, class SH>
__device__ __forceinline__ void pull_partials(const float* __restrict__ sm, int tx, int tz, float aS[3], float aW[3]) {
    constexpr int kNH = SH::kNH;
    constexpr int NX = D == 0 ? 2 : 3, NY = D == 1 ? 2 : 3, NZ = D == 2 ? 2 : 3;
#pragma unroll
    for(int izc = 0; izc < NZ; ++izc) {        // cell z = face z - 1 + izc
        const int oz = 1 - izc;                  // face offset from that cell
        const int iz = D == 2 ? oz : oz + 1;
#pragma unroll
        for(int ixc = 0; ixc < NX; ++ixc) {
            const int ox = 1 - ixc;
            const int ix = D == 0 ? ox : ox + 1;
            const int h = (tz + izc) * kHX + (tx + ixc);
#pragma unroll
            for(int j = (D == 1 ? 1 : 0); j < 3; ++j) {
                const int oy = j - 1;
                const int iy = D == 1 ? oy : oy + 1;
                const int s = (ix * NY + iy) * NZ + iz;
                aS[j] = aS[j] + sm[(2 * s) * kNH + h];
                aW[j] = aW[j] + sm[(2 * s + 1) * kNH + h];
            }
        }
    }
}

// Minimum squared distance from the particles of halo cell h (layer cy) to the centres of
// the 27 cells around it.  EXACT (some particle left the grid, so the whole launch takes
// it): a particle outside the grid (sorted into the clamped cell) reaches only the clamped
// 3x3x3 range of its own cell (PIC_Solver.cpp:633-635); otherwise every particle reaches
// all 27 and no per-slot test runs.
template<class SH, bool EXACT>
__device__ __forceinline__ void sdf_partials(const TileArgs& a, int x0, int z0, int cy, int h, uint32_t b,
                                             uint32_t e, float* __restrict__ sm) {
    constexpr int kNH = SH::kNH;
    const float inf = __int_as_float(0x7f800000);
    float m[27];
#pragma unroll
    for(int s = 0; s < 27; ++s) m[s] = inf;
    const GridDesc& g = a.g;
    const int cx = x0 - 1 + h % kHX, cz = z0 - 1 + h / kHX;
    if(b < e) {
        const float4* __restrict__ pos = a.rec + 3 * a.stride;
        // Grid::getWorldCoordinate(i + 0.5, ...) (Grid.h:186-194) of the 27 target cells
        float sx[3], sy[3], sz[3];
#pragma unroll
        for(int o = 0; o < 3; ++o) {
            sx[o] = ((float)(cx - 1 + o) + 0.5f) * g.dx + g.bmin[0];
            sy[o] = ((float)(cy - 1 + o) + 0.5f) * g.dx + g.bmin[1];
            sz[o] = ((float)(cz - 1 + o) + 0.5f) * g.dx + g.bmin[2];
        }
        float4 Ln = b < e ? __ldg(pos + b) : make_float4(0.f, 0.f, 0.f, 0.f);
        for(uint32_t q = b; q < e; ++q) {
            const float4 L = Ln;
            if(q + 1 < e) Ln = __ldg(pos + q + 1);
            float dxx[3], dyy[3], dzz[3];
#pragma unroll
            for(int o = 0; o < 3; ++o) {
                const float ddx = sx[o] - L.x, ddy = sy[o] - L.y, ddz = sz[o] - L.z;
                dxx[o] = ddx * ddx;
                dyy[o] = ddy * ddy;
                dzz[o] = ddz * ddz;
            }
            bool okx[3] = {true, true, true}, oky[3] = {true, true, true}, okz[3] = {true, true, true};
            if constexpr(EXACT) {
                const int ci = (int)((L.x - g.bmin[0]) / g.dx);
                const int cj = (int)((L.y - g.bmin[1]) / g.dx);
                const int ck = (int)((L.z - g.bmin[2]) / g.dx);
#pragma unroll
                for(int o = 0; o < 3; ++o) {
                    const int tx = cx - 1 + o, ty = cy - 1 + o, tz = cz - 1 + o;
                    okx[o] = !(tx < max(ci - 1, 0) || tx > min(ci + 1, g.G[0] - 1));
                    oky[o] = !(ty < max(cj - 1, 0) || ty > min(cj + 1, g.G[1] - 1));
                    okz[o] = !(tz < max(ck - 1, 0) || tz > min(ck + 1, g.G[2] - 1));
                }
            }
#pragma unroll
            for(int iz = 0; iz < 3; ++iz)
#pragma unroll
                for(int iy = 0; iy < 3; ++iy)
#pragma unroll
                    for(int ix = 0; ix < 3; ++ix) {
                        const float d2 = (dxx[ix] + dyy[iy]) + dzz[iz];  // glm::length2: (x*x + y*y) + z*z
                        const int s = (iz * 3 + iy) * 3 + ix;
                        if constexpr(EXACT) m[s] = fminf(m[s], (okx[ix] && oky[iy] && okz[iz]) ? d2 : inf);
                        else m[s] = fminf(m[s], d2);
                    }
        }
    }
#pragma unroll
    for(int s = 0; s < 27; ++s) sm[s * kNH + h] = m[s];
}

// Cell (x0 + tx, cy - 1 + j, z0 + tz) takes the minimum over its 9 neighbours of this layer.
template<class SH>
__device__ __forceinline__ void pull_sdf(const float* __restrict__ sm, int tx, int tz, float aM[3]) {
    constexpr int kNH = SH::kNH;
#pragma unroll
    for(int izc = 0; izc < 3; ++izc)
#pragma unroll
        for(int ixc = 0; ixc < 3; ++ixc) {
            const int h = (tz + izc) * kHX + (tx + ixc);
            const int ix = 2 - ixc, iz = 2 - izc;  // offset (target - source) + 1
#pragma unroll
            for(int j = 0; j < 3; ++j) {
                const int s = (iz * 3 + j) * 3 + ix;
                aM[j] = fminf(aM[j], sm[s * kNH + h]);
            }
        }
}

template<int D>
__device__ __forceinline__ void write_face(const TileArgs& a, int fx, int fy, int fz, float S, float W) {
    const int sx = a.g.G[0] + (D == 0), sy = a.g.G[1] + (D == 1), sz = a.g.G[2] + (D == 2);
    if(fx >= sx || fy >= sy || fz < 0 || fz >= sz) return;
    const size_t f = ((size_t)fz * sy + fy) * sx + fx;
    const bool ok = W > FLT_MIN;
    a.out[D][f] = ok ? S / W : S;
    a.valid[D][f] = ok ? 1 : 0;
}

__device__ __forceinline__ void write_phi(const TileArgs& a, int fx, int fy, int fz, float m) {
    const GridDesc& g = a.g;
    if(fx >= g.G[0] || fy >= g.G[1] || fz < 0 || fz >= g.G[2]) return;
    const float empty = g.dx * 3.0f;
    float ph = empty;
    if(m != __int_as_float(0x7f800000)) {
        const float val = sqrtf(m) - g.sdfRadius;
        if(val < ph) ph = val;
    }
    a.phi[((size_t)fz * g.G[1] + fy) * g.G[0] + fx] = ph;
}
} // namespace

// P2G: the three face components and the fluid SDF (FLIP); otherwise the fluid SDF alone.
// Which tile a block works on: its own launch's block index, or one given to it (a scene's
// tile in a batched launch).  Reading blockIdx keeps the indices out of registers.
struct OwnTile {
    __device__ __forceinline__ unsigned x() const { return blockIdx.x; }
    __device__ __forceinline__ unsigned z() const { return blockIdx.y; }
    __device__ __forceinline__ unsigned y() const { return blockIdx.z; }
};
struct GivenTile {
    unsigned bx, bz, by;
    __device__ __forceinline__ unsigned x() const { return bx; }
    __device__ __forceinline__ unsigned z() const { return bz; }
    __device__ __forceinline__ unsigned y() const { return by; }
};

// One block of the pass: tile (x, z) of face columns, y-chunk y.  EXACT: some particle
// left the grid (the same for the whole launch; see sdf_partials).  AFF: APIC / AFLIP
// momentum (cell_partials).
template<bool P2G, class SH, bool EXACT, bool AFF = false, class Tile>
__device__ __forceinline__ void tile_body(const TileArgs& a, const Tile tile) {
    constexpr int kTZ = SH::kTZ, kYC = SH::kYC;
    extern __shared__ float sm[];
    const GridDesc& g = a.g;
    const int t = threadIdx.y * kHX + threadIdx.x;        // this thread's halo cell
    const int tx = threadIdx.x - 1, tz = threadIdx.y - 1;  // interior column (faces) or halo
    const bool owner = tx >= 0 && tx < kTX && tz >= 0 && tz < kTZ;
    const int x0 = (int)tile.x() * kTX, z0 = (int)tile.z() * kTZ;
    const int yA = (int)tile.y() * kYC, yB = min(yA + kYC, g.G[1] + 1);  // face layers [yA, yB)
    const int fx = owner ? x0 + tx : INT_MAX, fz = owner ? z0 + tz : INT_MAX;
    {
        const int lo[3] = {x0 - 1, yA - 1, z0 - 1}, hi[3] = {x0 + kTX, yB, z0 + kTZ};
        if(!meets_particles(a.st, lo, hi)) {
            // no particle reaches the tile: empty faces and cells
            for(int fy = yA; fy < yB; ++fy) {
                if constexpr(P2G) {
                    write_face<0>(a, fx, fy, fz, 0.0f, 0.0f);
                    write_face<1>(a, fx, fy, fz, 0.0f, 0.0f);
                    write_face<2>(a, fx, fy, fz, 0.0f, 0.0f);
                }
                write_phi(a, fx, fy, fz, __int_as_float(0x7f800000));
            }
            return;
        }
    }
    const float inf = __int_as_float(0x7f800000);
    // accumulators of face layers cy - 1 + j (v, whose own axis is the walk, uses j = 1, 2)
    float uS[3] = {0.f, 0.f, 0.f}, uW[3] = {0.f, 0.f, 0.f};
    float vS[3] = {0.f, 0.f, 0.f}, vW[3] = {0.f, 0.f, 0.f};
    float wS[3] = {0.f, 0.f, 0.f}, wW[3] = {0.f, 0.f, 0.f};
    float aM[3] = {inf, inf, inf};
    for(int cy = yA - 1; cy <= yB; ++cy) {
        if(cy >= 0 && cy < g.G[1]) {
            uint32_t pb, pe;
            cell_range(a, x0, z0, cy, t, pb, pe);
            if constexpr(P2G) {
                cell_partials<0, SH, AFF>(a, t, pb, pe, sm, x0, z0, cy);
                __syncthreads();
                if(owner) pull_partials<0, SH>(sm, tx, tz, uS, uW);
                __syncthreads();
                if(cy < yB) {
                    cell_partials<1, SH, AFF>(a, t, pb, pe, sm, x0, z0, cy);
                    __syncthreads();
                    if(owner) pull_partials<1, SH>(sm, tx, tz, vS, vW);
                    __syncthreads();
                }
                cell_partials<2, SH, AFF>(a, t, pb, pe, sm, x0, z0, cy);
                __syncthreads();
                if(owner) pull_partials<2, SH>(sm, tx, tz, wS, wW);
                __syncthreads();
            }
            sdf_partials<SH, EXACT>(a, x0, z0, cy, t, pb, pe, sm);
            __syncthreads();
            if(owner) pull_sdf<SH>(sm, tx, tz, aM);
            __syncthreads();
        }
        // face / cell layer cy - 1 is complete for u, w and the SDF, face layer cy for v
        if(cy - 1 >= yA && cy - 1 < yB) {
            if constexpr(P2G) {
                write_face<0>(a, fx, cy - 1, fz, uS[0], uW[0]);
                write_face<2>(a, fx, cy - 1, fz, wS[0], wW[0]);
            }
            write_phi(a, fx, cy - 1, fz, aM[0]);
        }
        if constexpr(P2G) {
            if(cy >= yA && cy < yB) write_face<1>(a, fx, cy, fz, vS[1], vW[1]);
        }
        uS[0] = uS[1]; uS[1] = uS[2]; uS[2] = 0.f;
        uW[0] = uW[1]; uW[1] = uW[2]; uW[2] = 0.f;
        wS[0] = wS[1]; wS[1] = wS[2]; wS[2] = 0.f;
        wW[0] = wW[1]; wW[1] = wW[2]; wW[2] = 0.f;
        vS[1] = vS[2]; vS[2] = 0.f;
        vW[1] = vW[2]; vW[2] = 0.f;
        aM[0] = aM[1]; aM[1] = aM[2]; aM[2] = inf;
    }
}
// The rare launch in which some particle left the grid, kept out of line so that its
// per-slot tests do not weigh on the registers of the common path
template<bool P2G, class SH, bool AFF, class Tile>
__device__ __noinline__ void tile_body_exact(const TileArgs& a, const Tile tile) {
    tile_body<P2G, SH, true, AFF>(a, tile);
}
template<bool P2G, class SH, bool AFF = false>
__global__ void __launch_bounds__(SH::kThreads, SH::kMinBlocks) k_p2g_sdf_tile(const __grid_constant__ TileArgs a) {
    if((a.st->flags & BNN_FLAG_OUT_OF_GRID) != 0u) tile_body_exact<P2G, SH, AFF>(a, OwnTile{});
    else tile_body<P2G, SH, false, AFF>(a, OwnTile{});
}

// Batched: the tiles of all scenes of a batch in one launch (P: per-scene tile prefix);
// a block's flat tile index within its scene maps to (x, z, y) as in tile_grid
template<class SH>
__global__ void __launch_bounds__(SH::kThreads, SH::kMinBlocks) kb_p2g_sdf_tile(const TileArgs* __restrict__ A,
                                                                            const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const TileArgs& a = A[q];
    const unsigned gx = (unsigned)((a.g.G[0] + 1 + kTX - 1) / kTX);
    const unsigned gz = (unsigned)((a.g.G[2] + 1 + SH::kTZ - 1) / SH::kTZ);
    const GivenTile tile{b.x % gx, (b.x / gx) % gz, b.x / (gx * gz)};
    if((a.st->flags & BNN_FLAG_OUT_OF_GRID) != 0u) tile_body_exact<true, SH, false>(a, tile);  // the scene's flag
    else tile_body<true, SH, false, false>(a, tile);
}
static_assert(kHX == 32, "a warp is one row of halo cells");

template<class SH> static dim3 tile_grid_of(const GridDesc& g) {
    return dim3((unsigned)((g.G[0] + 1 + kTX - 1) / kTX), (unsigned)((g.G[2] + 1 + SH::kTZ - 1) / SH::kTZ),
                (unsigned)((g.G[1] + 1 + SH::kYC - 1) / SH::kYC));
}

// The dynamic shared memory above the 48 KB default is opted into once per kernel and device
template<class K> static void opt_in_smem(K* kern, size_t bytes, std::atomic<uint64_t>& configured) {
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if(!(configured.load(std::memory_order_acquire) & bit)) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        configured.fetch_or(bit, std::memory_order_acq_rel);
    }
}
template<bool P2G, class SH> static void launch_tile_sh(const TileArgs& a, cudaStream_t s) {
    static std::atomic<uint64_t> configured{0};
    opt_in_smem(k_p2g_sdf_tile<P2G, SH>, SH::kSmemBytes, configured);
    k_p2g_sdf_tile<P2G, SH><<<tile_grid_of<SH>(a.g), dim3(kHX, SH::kHZ), SH::kSmemBytes, s>>>(a);
    bnn_note_launch();
}
template<class SH>
static void launch_batch_sh(const TileArgs* A, const unsigned* P, int ns, unsigned tiles, cudaStream_t s) {
    static std::atomic<uint64_t> configured{0};
    opt_in_smem(kb_p2g_sdf_tile<SH>, SH::kSmemBytes, configured);
    kb_p2g_sdf_tile<SH><<<tiles, dim3(kHX, SH::kHZ), SH::kSmemBytes, s>>>(A, P, ns);
    bnn_note_launch();
}

// ---- shapes and their tuner -----------------------------------------------------------
// The tuner times every shape on the live pass the first time it meets a kind of launch
// (a resolution bucket of a lone scene: ceil((G + 1) / 32) cells per axis; for a batch, the
// scene count and total cells in powers of two) and keeps the fastest for it.  The pass is
// a pure function of the sorted particles (it writes every face and cell of its outputs and
// reads none of them), so the timing runs leave exactly what one run leaves, and since all
// shapes give the same bits the choice never changes a result.
constexpr int kShapeDims[kTileShapes][2] = {{S0::kTZ, S0::kYC}, {S1::kTZ, S1::kYC}, {S2::kTZ, S2::kYC},
                                            {S3::kTZ, S3::kYC}, {S4::kTZ, S4::kYC}, {S5::kTZ, S5::kYC}};

static dim3 tile_grid(const GridDesc& g, int shape) {
    switch(shape) {
    case 1: return tile_grid_of<S1>(g);
    case 2: return tile_grid_of<S2>(g);
    case 3: return tile_grid_of<S3>(g);
    case 4: return tile_grid_of<S4>(g);
    case 5: return tile_grid_of<S5>(g);
    default: return tile_grid_of<S0>(g);
    }
}
static void launch_p2g_shape(int shape, const TileArgs& a, cudaStream_t s) {
    switch(shape) {
    case 1: launch_tile_sh<true, S1>(a, s); break;
    case 2: launch_tile_sh<true, S2>(a, s); break;
    case 3: launch_tile_sh<true, S3>(a, s); break;
    case 4: launch_tile_sh<true, S4>(a, s); break;
    case 5: launch_tile_sh<true, S5>(a, s); break;
    default: launch_tile_sh<true, S0>(a, s); break;
    }
}
static void launch_batch_shape(int shape, const TileArgs* A, const unsigned* P, int ns, unsigned tiles, cudaStream_t s) {
    if(tiles == 0) return;
    switch(shape) {
    case 1: launch_batch_sh<S1>(A, P, ns, tiles, s); break;
    case 2: launch_batch_sh<S2>(A, P, ns, tiles, s); break;
    case 3: launch_batch_sh<S3>(A, P, ns, tiles, s); break;
    case 4: launch_batch_sh<S4>(A, P, ns, tiles, s); break;
    case 5: launch_batch_sh<S5>(A, P, ns, tiles, s); break;
    default: launch_batch_sh<S0>(A, P, ns, tiles, s); break;
    }
}

namespace {
struct TuneEntry {
    int shape = 0;
    float us[kTileShapes] = {};
};
struct Tuner {
    std::mutex mu;
    std::map<uint64_t, TuneEntry> table;
    int forced = -1;  // bnn_set_tile_shape
};
Tuner& tuner() {
    static Tuner t;
    return t;
}
inline uint64_t log2_bucket(uint64_t x) {
    uint64_t b = 0;
    while((1ull << b) < x && b < 63) ++b;
    return b;
}
uint64_t scene_key(const GridDesc& g) {
    int dev = 0;
    cudaGetDevice(&dev);
    uint64_t k = (uint64_t)(dev & 0xff) << 56;
    for(int a = 0; a < 3; ++a) k |= (uint64_t)(((g.G[a] + 1 + 31) / 32) & 0xffff) << (16 * a);
    return k;
}
// The shape for key, or -1 when it still has to be tuned
int lookup(uint64_t key) {
    Tuner& t = tuner();
    std::lock_guard<std::mutex> lk(t.mu);
    if(t.forced >= 0) return t.forced;
    auto it = t.table.find(key);
    return it == t.table.end() ? -1 : it->second.shape;
}
// Times launch(shape) for every shape (best of two rounds) on stream s and records the
// fastest under key (the default unless another is 3% faster); the stream is synchronised.
template<class F> int tune(uint64_t key, cudaStream_t s, F launch) {
    constexpr int kRounds = 2;
    cudaEvent_t ev[kRounds][kTileShapes + 1];
    for(auto& r : ev)
        for(auto& e : r) cudaEventCreate(&e);
    for(int r = 0; r < kRounds; ++r) {
        cudaEventRecord(ev[r][0], s);
        for(int v = 0; v < kTileShapes; ++v) {
            launch(v);
            cudaEventRecord(ev[r][v + 1], s);
        }
    }
    cudaEventSynchronize(ev[kRounds - 1][kTileShapes]);
    TuneEntry e;
    for(int v = 0; v < kTileShapes; ++v) {
        float best = FLT_MAX;
        for(int r = 0; r < kRounds; ++r) {
            float ms = FLT_MAX;
            if(cudaEventElapsedTime(&ms, ev[r][v], ev[r][v + 1]) != cudaSuccess) ms = FLT_MAX;
            best = ms < best ? ms : best;
        }
        e.us[v] = best * 1000.f;
        if(e.us[v] < e.us[e.shape]) e.shape = v;
    }
    // timings this close are noise: another shape must beat the default by 3%
    if(e.us[e.shape] > 0.97f * e.us[0]) e.shape = 0;
    for(auto& r : ev)
        for(auto& ee : r) cudaEventDestroy(ee);
    Tuner& t = tuner();
    std::lock_guard<std::mutex> lk(t.mu);
    t.table[key] = e;
    return e.shape;
}
} // namespace

int tile_shape_set(int shape) {
    if(shape < -1 || shape >= kTileShapes) return BNN_ERR_INVALID_ARGUMENT;
    Tuner& t = tuner();
    std::lock_guard<std::mutex> lk(t.mu);
    t.forced = shape;
    return BNN_OK;
}
void tile_shape_dims(int shape, int* tz, int* yc) {
    *tz = kShapeDims[shape][0];
    *yc = kShapeDims[shape][1];
}
// One JSON object per tuned launch kind, one per line
std::string tile_tuning_report() {
    Tuner& t = tuner();
    std::lock_guard<std::mutex> lk(t.mu);
    std::string out;
    char buf[512];
    for(const auto& kv : t.table) {
        const uint64_t k = kv.first;
        const bool batch = (k >> 48) & 1;
        int n = 0;
        if(batch)
            n = std::snprintf(buf, sizeof buf, "{\"kind\": \"batch\", \"scenes_le\": %llu, \"cells_le\": %llu",
                              1ull << ((k >> 24) & 0x3f), 1ull << (k & 0x3f));
        else
            n = std::snprintf(buf, sizeof buf, "{\"kind\": \"scene\", \"cells_per_axis_le\": [%d, %d, %d]",
                              (int)(k & 0xffff) * 32 - 1, (int)((k >> 16) & 0xffff) * 32 - 1,
                              (int)((k >> 32) & 0xffff) * 32 - 1);
        out.append(buf, (size_t)n);
        const int sh = kv.second.shape;
        n = std::snprintf(buf, sizeof buf, ", \"shape\": %d, \"tz\": %d, \"yc\": %d, \"us\": [", sh, kShapeDims[sh][0],
                          kShapeDims[sh][1]);
        out.append(buf, (size_t)n);
        for(int v = 0; v < kTileShapes; ++v) {
            n = std::snprintf(buf, sizeof buf, "%s%.1f", v ? ", " : "", kv.second.us[v]);
            out.append(buf, (size_t)n);
        }
        out += "]}\n";
    }
    return out;
}

// FLIP P2G of the three components together with the fluid SDF
void launch_p2g_sdf(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                    size_t stride, float* const* out, uint8_t* const* valid, float* phi, cudaStream_t s) {
    const TileArgs a{g, st, cellStart, rec, stride, {out[0], out[1], out[2]}, {valid[0], valid[1], valid[2]}, phi};
    const uint64_t key = scene_key(g);
    int shape = lookup(key);
    if(shape < 0) shape = tune(key, s, [&](int v) { launch_p2g_shape(v, a, s); });
    else launch_p2g_shape(shape, a, s);
}

// APIC / AFLIP: the same pass with the affine momentum term (C9: the sorted particles'
// affine matrices), in the default tile shape
void launch_p2g_sdf_affine(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                           const float* C9, size_t stride, float* const* out, uint8_t* const* valid, float* phi,
                           cudaStream_t s) {
    const TileArgs a{g, st, cellStart, rec, stride, {out[0], out[1], out[2]}, {valid[0], valid[1], valid[2]}, phi, C9};
    static std::atomic<uint64_t> configured{0};
    opt_in_smem(k_p2g_sdf_tile<true, S0, true>, S0::kSmemBytes, configured);
    k_p2g_sdf_tile<true, S0, true><<<tile_grid_of<S0>(g), dim3(kHX, S0::kHZ), S0::kSmemBytes, s>>>(a);
    bnn_note_launch();
}

// Tiles of one scene's P2G + SDF pass in a shape (the batched launch's share of the scene)
unsigned p2g_sdf_tiles(const GridDesc& g, int shape) {
    const dim3 d = tile_grid(g, shape);
    return d.x * d.y * d.z;
}
// Size of the per-scene argument record the batched launch reads, and its host-side fill
size_t p2g_tile_args_bytes() { return sizeof(TileArgs); }
void p2g_tile_args(void* out, const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                   size_t stride, float* const U[3], uint8_t* const valid[3], float* phi) {
    TileArgs a{g, st, cellStart, rec, stride, {U[0], U[1], U[2]}, {valid[0], valid[1], valid[2]}, phi};
    memcpy(out, &a, sizeof a);
}
// The batch's P2G + SDF pass: P[shape] is the tile prefix of the scenes in that shape,
// tiles[shape] its total (host copy); tuned per batch kind like a lone scene's pass
static uint64_t batch_key(int ns, uint64_t cells) {
    int dev = 0;
    cudaGetDevice(&dev);
    return ((uint64_t)(dev & 0xff) << 56) | (1ull << 48) | (log2_bucket((uint64_t)ns) << 24) | log2_bucket(cells);
}
int p2g_batch_shape(int ns, uint64_t cells) {
    static std::atomic<uint64_t> c0{0}, c1{0}, c2{0}, c3{0}, c4{0}, c5{0};
    opt_in_smem(kb_p2g_sdf_tile<S0>, S0::kSmemBytes, c0);
    opt_in_smem(kb_p2g_sdf_tile<S1>, S1::kSmemBytes, c1);
    opt_in_smem(kb_p2g_sdf_tile<S2>, S2::kSmemBytes, c2);
    opt_in_smem(kb_p2g_sdf_tile<S3>, S3::kSmemBytes, c3);
    opt_in_smem(kb_p2g_sdf_tile<S4>, S4::kSmemBytes, c4);
    opt_in_smem(kb_p2g_sdf_tile<S5>, S5::kSmemBytes, c5);
    return lookup(batch_key(ns, cells));
}
void launch_p2g_sdf_batch(const void* args, const unsigned* const* P, const unsigned* tiles, int ns, uint64_t cells,
                          cudaStream_t s) {
    const uint64_t key = batch_key(ns, cells);
    const TileArgs* A = (const TileArgs*)args;
    int shape = lookup(key);
    if(shape < 0) shape = tune(key, s, [&](int v) { launch_batch_shape(v, A, P[v], ns, tiles[v], s); });
    else launch_batch_shape(shape, A, P[shape], ns, tiles[shape], s);
}

// The fluid SDF alone (APIC / AFLIP / PIC), in the default shape
void launch_fluid_sdf_tile(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                           size_t stride, float* phi, cudaStream_t s) {
    const TileArgs a{g, st, cellStart, rec, stride, {nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}, phi};
    launch_tile_sh<false, S0>(a, s);
}

} // namespace bnn
