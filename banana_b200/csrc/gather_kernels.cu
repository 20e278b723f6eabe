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
#include <climits>

namespace bnn {

namespace {
#ifndef BNN_TILE_Z
#define BNN_TILE_Z 6
#endif
#ifndef BNN_TILE_Y
#define BNN_TILE_Y 8
#endif
#ifndef BNN_TILE_MIN_BLOCKS
#define BNN_TILE_MIN_BLOCKS (768 / (32 * (BNN_TILE_Z + 2)))
#endif
// A thread per cell of the tile plus its 1-cell halo: a warp is one row of 32 cells along x
// (30 interior columns and one halo cell each side), kTZ + 2 rows along z.  Every thread
// forms the partials of exactly one cell, and the interior threads own the faces.
constexpr int kHX = 32, kTX = kHX - 2;      // cells per row, interior face columns along x
constexpr int kTZ = BNN_TILE_Z;              // interior face columns along z
constexpr int kHZ = kTZ + 2;
constexpr int kYC = BNN_TILE_Y;              // face layers per block along y (the walk)
constexpr int kThreads = kHX * kHZ;
constexpr int kNH = kHX * kHZ;               // cells of one layer whose partials the tile needs
constexpr int kPartials = 36;              // 18 face slots x (momentum, weight); the SDF has 27
constexpr size_t kSmemBytes = sizeof(float) * kPartials * kNH;

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

// Partials of component D for halo cell h of cell layer cy into sm (slot-major planes).
template<int D>
__device__ __forceinline__ void cell_partials(const TileArgs& a, int x0, int z0, int cy, int h, float* __restrict__ sm) {
    constexpr int NX = D == 0 ? 2 : 3, NY = D == 1 ? 2 : 3, NZ = D == 2 ? 2 : 3;
    constexpr int NS = NX * NY * NZ;
    float S[NS], W[NS];
#pragma unroll
    for(int s = 0; s < NS; ++s) { S[s] = 0.0f; W[s] = 0.0f; }
    const int cx = x0 - 1 + h % kHX, cz = z0 - 1 + h / kHX;
    if(cx >= 0 && cx < a.g.G[0] && cz >= 0 && cz < a.g.G[2]) {
        const size_t c = ((size_t)cz * a.g.G[1] + cy) * a.g.G[0] + cx;
        const uint32_t b = __ldg(a.cellStart + c), e = __ldg(a.cellStart + c + 1);
        const float4* __restrict__ recD = a.rec + (size_t)D * a.stride;
        for(uint32_t q = b; q < e; ++q) {
            const float4 L = __ldg(recD + q);
            float wx[NX], wy[NY], wz[NZ];
            if constexpr(D == 0) own_axis(L.x, wx); else side_axis(L.x, wx);
            if constexpr(D == 1) own_axis(L.y, wy); else side_axis(L.y, wy);
            if constexpr(D == 2) own_axis(L.z, wz); else side_axis(L.z, wz);
#pragma unroll
            for(int ix = 0; ix < NX; ++ix)
#pragma unroll
                for(int iy = 0; iy < NY; ++iy) {
                    const float wxy = wx[ix] * wy[iy];
#pragma unroll
                    for(int iz = 0; iz < NZ; ++iz) {
                        const int s = (ix * NY + iy) * NZ + iz;
                        const float w = wxy * wz[iz];
                        S[s] = S[s] + w * L.w;
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
template<int D>
__device__ __forceinline__ void pull_partials(const float* __restrict__ sm, int tx, int tz, float aS[3], float aW[3]) {
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
// the 27 cells around it.  exact: a particle outside the grid (sorted into the clamped
// cell) reaches only the clamped 3x3x3 range of its own cell (PIC_Solver.cpp:633-635).
__device__ __forceinline__ void sdf_partials(const TileArgs& a, int x0, int z0, int cy, int h, bool exact,
                                             float* __restrict__ sm) {
    const float inf = __int_as_float(0x7f800000);
    float m[27];
#pragma unroll
    for(int s = 0; s < 27; ++s) m[s] = inf;
    const GridDesc& g = a.g;
    const int cx = x0 - 1 + h % kHX, cz = z0 - 1 + h / kHX;
    if(cx >= 0 && cx < g.G[0] && cz >= 0 && cz < g.G[2]) {
        const size_t c = ((size_t)cz * g.G[1] + cy) * g.G[0] + cx;
        const uint32_t b = __ldg(a.cellStart + c), e = __ldg(a.cellStart + c + 1);
        const float4* __restrict__ pos = a.rec + 3 * a.stride;
        // Grid::getWorldCoordinate(i + 0.5, ...) (Grid.h:186-194) of the 27 target cells
        float sx[3], sy[3], sz[3];
#pragma unroll
        for(int o = 0; o < 3; ++o) {
            sx[o] = ((float)(cx - 1 + o) + 0.5f) * g.dx + g.bmin[0];
            sy[o] = ((float)(cy - 1 + o) + 0.5f) * g.dx + g.bmin[1];
            sz[o] = ((float)(cz - 1 + o) + 0.5f) * g.dx + g.bmin[2];
        }
        for(uint32_t q = b; q < e; ++q) {
            const float4 L = __ldg(pos + q);
            float dxx[3], dyy[3], dzz[3];
#pragma unroll
            for(int o = 0; o < 3; ++o) {
                const float ddx = sx[o] - L.x, ddy = sy[o] - L.y, ddz = sz[o] - L.z;
                dxx[o] = ddx * ddx;
                dyy[o] = ddy * ddy;
                dzz[o] = ddz * ddz;
            }
            bool okx[3] = {true, true, true}, oky[3] = {true, true, true}, okz[3] = {true, true, true};
            if(exact) {
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
                        m[s] = fminf(m[s], (okx[ix] && oky[iy] && okz[iz]) ? d2 : inf);
                    }
        }
    }
#pragma unroll
    for(int s = 0; s < 27; ++s) sm[s * kNH + h] = m[s];
}

// Cell (x0 + tx, cy - 1 + j, z0 + tz) takes the minimum over its 9 neighbours of this layer.
__device__ __forceinline__ void pull_sdf(const float* __restrict__ sm, int tx, int tz, float aM[3]) {
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
template<bool P2G>
__global__ void __launch_bounds__(kThreads, BNN_TILE_MIN_BLOCKS) k_p2g_sdf_tile(TileArgs a) {
    extern __shared__ float sm[];
    const GridDesc& g = a.g;
    const int t = threadIdx.y * kHX + threadIdx.x;        // this thread's halo cell
    const int tx = threadIdx.x - 1, tz = threadIdx.y - 1;  // interior column (faces) or halo
    const bool owner = tx >= 0 && tx < kTX && tz >= 0 && tz < kTZ;
    const int x0 = blockIdx.x * kTX, z0 = blockIdx.y * kTZ;
    const int yA = blockIdx.z * kYC, yB = min(yA + kYC, g.G[1] + 1);  // face layers [yA, yB)
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
    const bool exact = (a.st->flags & BNN_FLAG_OUT_OF_GRID) != 0u;
    const float inf = __int_as_float(0x7f800000);
    // accumulators of face layers cy - 1 + j (v, whose own axis is the walk, uses j = 1, 2)
    float uS[3] = {0.f, 0.f, 0.f}, uW[3] = {0.f, 0.f, 0.f};
    float vS[3] = {0.f, 0.f, 0.f}, vW[3] = {0.f, 0.f, 0.f};
    float wS[3] = {0.f, 0.f, 0.f}, wW[3] = {0.f, 0.f, 0.f};
    float aM[3] = {inf, inf, inf};
    for(int cy = yA - 1; cy <= yB; ++cy) {
        if(cy >= 0 && cy < g.G[1]) {
            if constexpr(P2G) {
                cell_partials<0>(a, x0, z0, cy, t, sm);
                __syncthreads();
                if(owner) pull_partials<0>(sm, tx, tz, uS, uW);
                __syncthreads();
                if(cy < yB) {
                    cell_partials<1>(a, x0, z0, cy, t, sm);
                    __syncthreads();
                    if(owner) pull_partials<1>(sm, tx, tz, vS, vW);
                    __syncthreads();
                }
                cell_partials<2>(a, x0, z0, cy, t, sm);
                __syncthreads();
                if(owner) pull_partials<2>(sm, tx, tz, wS, wW);
                __syncthreads();
            }
            sdf_partials(a, x0, z0, cy, t, exact, sm);
            __syncthreads();
            if(owner) pull_sdf(sm, tx, tz, aM);
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

static dim3 tile_grid(const GridDesc& g) {
    return dim3((unsigned)((g.G[0] + 1 + kTX - 1) / kTX), (unsigned)((g.G[2] + 1 + kTZ - 1) / kTZ),
                (unsigned)((g.G[1] + 1 + kYC - 1) / kYC));
}
static_assert(kHX == 32, "a warp is one row of halo cells");

// The dynamic shared memory above the 48 KB default is opted into once per device.
template<bool P2G>
static void launch_tile(const TileArgs& a, cudaStream_t s) {
    static std::atomic<uint64_t> configured{0};  // bit per device ordinal
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if(!(configured.load(std::memory_order_acquire) & bit)) {
        cudaFuncSetAttribute(k_p2g_sdf_tile<P2G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
        configured.fetch_or(bit, std::memory_order_acq_rel);
    }
    k_p2g_sdf_tile<P2G><<<tile_grid(a.g), dim3(kHX, kHZ), kSmemBytes, s>>>(a);
    bnn_note_launch();
}

// FLIP P2G of the three components together with the fluid SDF
void launch_p2g_sdf(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                    size_t stride, float* const* out, uint8_t* const* valid, float* phi, cudaStream_t s) {
    TileArgs a{g, st, cellStart, rec, stride, {out[0], out[1], out[2]}, {valid[0], valid[1], valid[2]}, phi};
    launch_tile<true>(a, s);
}

// The fluid SDF alone (APIC / AFLIP / PIC)
void launch_fluid_sdf_tile(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                           size_t stride, float* phi, cudaStream_t s) {
    TileArgs a{g, st, cellStart, rec, stride, {nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}, phi};
    launch_tile<false>(a, s);
}

} // namespace bnn
