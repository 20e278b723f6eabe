// Column gathers for P2G (non-affine) and the fluid SDF.
//
// Both read one 16-byte record per candidate particle, written by the sort's gather
// (flip_kernels.cu, k_gather_particles): the P2G stencil record of the component, or the
// position.  Tuned on B200 at 256^3 (12.7M particles): 32 x 8 threads per block, columns
// of 4 outputs, particle records loaded in aligned pairs (one 256-bit load per pair), a
// register budget for 4 blocks per SM (no spills).
//
// One thread owns a column of kCol consecutive outputs (faces of one component, or cells)
// along one axis, on one or two rows of the third axis; the 32 lanes of a warp own 32
// consecutive x positions, so their particle loads fall on a few cache lines.  A face or cell only receives from particles of the
// cells one step around it, so the thread walks the cell rows around its whole column
// once (kCol + 2 rows along the column axis instead of 3 per output) and hands every
// particle to the outputs of the column it can reach.  Rows are walked in linear cell
// order (z outer, y inner) and particles in sorted order inside a row, so every output
// sees its particles in exactly the order of the serial reference loop over cell-sorted
// particles: the sums are bit-identical to the per-output gathers in flip_kernels.cu.
//
// The fluid SDF keeps the minimum squared distance instead of the minimum distance:
// sqrtf (correctly rounded) and the subtraction of the particle radius are both
// non-decreasing, so min(sqrtf(d2) - r) == sqrtf(min d2) - r exactly, and one square root
// per cell replaces one per candidate particle.
//
// Thread blocks whose column box lies more than one cell away from every particle (the
// occupied-cell bounding box is reduced during advection) only write the empty values.
#include "bnn_internal.cuh"

namespace bnn {

namespace {
#ifndef BNN_COL_LEN
#define BNN_COL_LEN 4
#endif
#ifndef BNN_COL_ROWS
#define BNN_COL_ROWS 8
#endif
#ifndef BNN_P2G_RPT
#define BNN_P2G_RPT 1
#endif
#ifndef BNN_SDF_RPT
#define BNN_SDF_RPT 2
#endif
constexpr int kCol = BNN_COL_LEN;     // outputs per thread along the column axis
constexpr int kLx = 32;               // threads along x
constexpr int kLr = BNN_COL_ROWS;     // threads along the row axis
// outputs per thread along the row axis: the SDF's cheap candidates gain from sharing
// rows between two outputs, P2G's heavier ones do not
constexpr int kRptP2G = BNN_P2G_RPT;
constexpr int kRptSdf = BNN_SDF_RPT;

// Records q0 and q0 + 1 (q0 even) in one 256-bit load.  The record planes start on
// 32-byte boundaries (the particle capacity, their stride, is a multiple of 64) and hold
// two spare records past the last plane, so a pair never leaves the allocation.
__device__ __forceinline__ void ldg_pair(const float4* p, float4& a, float4& b) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// Does [lo, hi] (per axis) meet the occupied-cell box grown by one cell?
__device__ __forceinline__ bool near_particles(const DevState* st, const int lo[3], const int hi[3]) {
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const int bl = st->bbox[d], bh = st->bbox[3 + d];
        if(bh < bl) return false;  // no particles
        if(hi[d] < bl - 1 || lo[d] > bh + 1) return false;
    }
    return true;
}
} // namespace

// FLIP_Solver::mapParticles2Grid (FLIP_Solver.cpp:57-95) for component D.  The column axis
// is z for u and v faces and y for w faces (never the component's own axis); the other
// non-x axis is the thread-row axis.
template<int D>
__global__ void __launch_bounds__(kLx * kLr, 4) k_p2g_col(GridDesc g, const DevState* __restrict__ st,
                                                       const uint32_t* __restrict__ cellStart,
                                                       const float4* __restrict__ rec, size_t stride,
                                                       float* __restrict__ out, uint8_t* __restrict__ valid) {
    constexpr int A = (D == 2) ? 1 : 2;  // column axis
    constexpr int R = (D == 2) ? 2 : 1;  // thread-row axis
    const int sz[3] = {g.G[0] + (D == 0), g.G[1] + (D == 1), g.G[2] + (D == 2)};
    const int i = blockIdx.x * kLx + threadIdx.x;
    const int r0 = (blockIdx.y * kLr + threadIdx.y) * kRptP2G;  // rows r0 .. r0 + kRptP2G - 1
    const int a0 = blockIdx.z * kCol;
    auto face_index = [&](int ur, int u) {
        const int r = r0 + ur;
        const int fy = (A == 1) ? a0 + u : r, fz = (A == 2) ? a0 + u : r;
        return ((size_t)fz * sz[1] + fy) * sz[0] + i;
    };
    {
        int lo[3], hi[3];
        lo[0] = blockIdx.x * kLx; hi[0] = lo[0] + kLx - 1;
        lo[R] = blockIdx.y * kLr * kRptP2G; hi[R] = lo[R] + kLr * kRptP2G - 1;
        lo[A] = a0; hi[A] = a0 + kCol - 1;
        if(!near_particles(st, lo, hi)) {
            if(i < sz[0]) {
#pragma unroll
                for(int ur = 0; ur < kRptP2G; ++ur)
#pragma unroll
                    for(int u = 0; u < kCol; ++u)
                        if(r0 + ur < sz[R] && a0 + u < sz[A]) { out[face_index(ur, u)] = 0.f; valid[face_index(ur, u)] = 0; }
            }
            return;
        }
    }
    float S[kRptP2G][kCol], W[kRptP2G][kCol];
#pragma unroll
    for(int ur = 0; ur < kRptP2G; ++ur)
#pragma unroll
        for(int u = 0; u < kCol; ++u) { S[ur][u] = 0.f; W[ur][u] = 0.f; }
    const int xlo = max(i - 1, 0), xhi = min(D == 0 ? i : i + 1, g.G[0] - 1);
    const float4* __restrict__ recD = rec + (size_t)D * stride;

    // one cell row: A coordinate a0 - 1 + t, R coordinate r0 - 1 + dr.  A face at row
    // offset ur / column offset u is reached from rows dr in {ur, ur+1, ur+2} (one row
    // fewer along the component's own axis) and t in {u, u+1, u+2}.
    auto row = [&](int t, int dr) __attribute__((always_inline)) {
        const int ca = a0 - 1 + t, rr = r0 - 1 + dr;
        if(ca < 0 || ca > g.G[A] - 1 || rr < 0 || rr > g.G[R] - 1) return;
        if(xlo > xhi) return;
        const int kk = (A == 2) ? ca : rr, jj = (A == 1) ? ca : rr;
        const size_t base = ((size_t)kk * g.G[1] + jj) * g.G[0];
        // the row segment holds cells xlo..xhi (at most 3): c1, c2 split it by cell
        const uint32_t b = __ldg(cellStart + base + xlo), e = __ldg(cellStart + base + xhi + 1);
        const uint32_t c1 = __ldg(cellStart + base + min(xlo + 1, xhi + 1));
        const uint32_t c2 = __ldg(cellStart + base + min(xlo + 2, xhi + 1));
        // Particles are taken in aligned pairs (one 256-bit load; the pair may start one
        // record before b and end one after e - 1, those slots being masked).  A particle
        // that does not reach an output adds +0 to its sums, which leaves them unchanged
        // (they start at +0 and can never become -0), so no branch is needed.
        for(uint32_t q0 = b & ~1u; q0 < e; q0 += 2) {
            float4 L[2];
            ldg_pair(recD + q0, L[0], L[1]);
#pragma unroll
            for(int w = 0; w < 2; ++w) {
                const uint32_t q = q0 + (uint32_t)w;
                const int cx = xlo + (q >= c1 ? 1 : 0) + (q >= c2 ? 1 : 0);
                const float ex = L[w].x, ey = L[w].y, ez = L[w].z;
                const float eR = (R == 1) ? ey : ez, eA = (A == 1) ? ey : ez;
                // sign bit set: stencil base = cell - 1
                const int si = cx + (__float_as_int(ex) >> 31);
                const int sr = rr + (__float_as_int(eR) >> 31);
                const int sa = ca + (__float_as_int(eA) >> 31);
                const float fi = fabsf(ex), fr = fabsf(eR), fa = fabsf(eA);
                const bool reach = (q >= b && q < e) && (si == i || si == i - 1);
                const float wx = (si == i) ? (1.0f - fi) : fi;
#pragma unroll
                for(int ddr = -2; ddr <= 0; ++ddr) {
                    const int ur = dr + ddr;
                    if(ur < 0 || ur >= kRptP2G) continue;
                    const int fr_ = r0 + ur;
                    const bool okR = reach && (sr == fr_ || sr == fr_ - 1);
                    const float wr = (sr == fr_) ? (1.0f - fr) : fr;
                    const float wxr = wx * wr;  // (wx * wy) when the column axis is z
#pragma unroll
                    for(int du = -1; du <= 1; ++du) {
                        const int u = t - 1 + du;
                        if(u < 0 || u >= kCol) continue;
                        const int fa_ = a0 + u;
                        const bool ok = okR && (sa == fa_ || sa == fa_ - 1);
                        const float wa = (sa == fa_) ? (1.0f - fa) : fa;
                        // weight = wx * wy * wz, multiplied left to right
                        const float wgt = (A == 2) ? wxr * wa : (wx * wa) * wr;
                        const float m = wgt * L[w].w;
                        S[ur][u] = S[ur][u] + (ok ? m : 0.f);
                        W[ur][u] = W[ur][u] + (ok ? wgt : 0.f);
                    }
                }
            }
        }
    };
    // rows in linear cell order: z outer, y inner
    constexpr int NR = kRptP2G + (R == D ? 1 : 2);  // row offsets dr = 0 .. NR-1
    if(A == 2) {
#pragma unroll
        for(int t = 0; t < kCol + 2; ++t)
#pragma unroll
            for(int dr = 0; dr < NR; ++dr) row(t, dr);
    } else {
#pragma unroll
        for(int dr = 0; dr < NR; ++dr)
#pragma unroll
            for(int t = 0; t < kCol + 2; ++t) row(t, dr);
    }
    if(i < sz[0]) {
#pragma unroll
        for(int ur = 0; ur < kRptP2G; ++ur)
#pragma unroll
            for(int u = 0; u < kCol; ++u) {
                if(r0 + ur >= sz[R] || a0 + u >= sz[A]) continue;
                const bool ok = W[ur][u] > FLT_MIN;
                out[face_index(ur, u)] = ok ? S[ur][u] / W[ur][u] : S[ur][u];
                valid[face_index(ur, u)] = ok ? 1 : 0;
            }
    }
}

// PIC_Solver::computeFluidSDF (PIC_Solver.cpp:601-652): phi of a cell = min(3 dx,
// min over the particles whose clamped 3x3x3 cell range holds it of |x_cell - x_p| - r).
// The column axis is z.  The range test against the particle's own cell only matters for
// a particle outside the grid (its own cell differs from the clamped cell it is sorted
// into); the advection flags that case and the test is then made for every candidate.
__global__ void __launch_bounds__(kLx * kLr, 4) k_fluid_sdf_col(GridDesc g, const DevState* __restrict__ st,
                                                             const uint32_t* __restrict__ cellStart,
                                                             const float4* __restrict__ pos, float* __restrict__ phi) {
    const int i = blockIdx.x * kLx + threadIdx.x;
    const int j0 = (blockIdx.y * kLr + threadIdx.y) * kRptSdf;  // cells j0 .. j0 + kRptSdf - 1
    const int k0 = blockIdx.z * kCol;
    const float empty = g.dx * 3.0f;
    auto cell_index = [&](int uj, int u) { return ((size_t)(k0 + u) * g.G[1] + (j0 + uj)) * g.G[0] + i; };
    {
        const int lo[3] = {(int)(blockIdx.x * kLx), (int)(blockIdx.y * kLr * kRptSdf), k0};
        const int hi[3] = {lo[0] + kLx - 1, lo[1] + kLr * kRptSdf - 1, k0 + kCol - 1};
        if(!near_particles(st, lo, hi)) {
            if(i < g.G[0]) {
#pragma unroll
                for(int uj = 0; uj < kRptSdf; ++uj)
#pragma unroll
                    for(int u = 0; u < kCol; ++u)
                        if(j0 + uj < g.G[1] && k0 + u < g.G[2]) phi[cell_index(uj, u)] = empty;
            }
            return;
        }
    }
    const bool exact = (st->flags & BNN_FLAG_OUT_OF_GRID) != 0u;
    const float inf = __int_as_float(0x7f800000);
    // Grid::getWorldCoordinate(i + 0.5, j + 0.5, k + 0.5) (Grid.h:186-194)
    const float sxw = ((float)i + 0.5f) * g.dx + g.bmin[0];
    float m[kRptSdf][kCol];
#pragma unroll
    for(int uj = 0; uj < kRptSdf; ++uj)
#pragma unroll
        for(int u = 0; u < kCol; ++u) m[uj][u] = inf;
    const int xlo = max(i - 1, 0), xhi = min(i + 1, g.G[0] - 1);
#pragma unroll
    for(int t = 0; t < kCol + 2; ++t) {
        const int kk = k0 - 1 + t;
        if(kk < 0 || kk > g.G[2] - 1) continue;
#pragma unroll
        for(int dj = 0; dj < kRptSdf + 2; ++dj) {
            const int jj = j0 - 1 + dj;
            if(jj < 0 || jj > g.G[1] - 1 || xlo > xhi) continue;
            const size_t base = ((size_t)kk * g.G[1] + jj) * g.G[0];
            const uint32_t b = __ldg(cellStart + base + xlo), e = __ldg(cellStart + base + xhi + 1);
            for(uint32_t q0 = b & ~1u; q0 < e; q0 += 2) {
                float4 L[2];
                ldg_pair(pos + q0, L[0], L[1]);
#pragma unroll
                for(int w = 0; w < 2; ++w) {
                    const float ddx = sxw - L[w].x;
                    const float dxx = ddx * ddx;
                    const uint32_t q = q0 + (uint32_t)w;
                    bool reach = q >= b && q < e;
                    int ci = 0, cj = 0, ck = 0;
                    if(exact) {
                        // the particle's own cell (Grid::getGridCoordinate, truncated) and its
                        // clamped 3x3x3 range (PIC_Solver.cpp:633-635)
                        ci = (int)((L[w].x - g.bmin[0]) / g.dx);
                        cj = (int)((L[w].y - g.bmin[1]) / g.dx);
                        ck = (int)((L[w].z - g.bmin[2]) / g.dx);
                        reach = reach && !(i < max(ci - 1, 0) || i > min(ci + 1, g.G[0] - 1));
                    }
#pragma unroll
                    for(int ddj = -2; ddj <= 0; ++ddj) {
                        const int uj = dj + ddj;
                        if(uj < 0 || uj >= kRptSdf) continue;
                        const int j = j0 + uj;
                        const float syw = ((float)j + 0.5f) * g.dx + g.bmin[1];
                        const float ddy = syw - L[w].y;
                        const float dxy = dxx + ddy * ddy;
                        const bool okJ = reach && !(exact && (j < max(cj - 1, 0) || j > min(cj + 1, g.G[1] - 1)));
#pragma unroll
                        for(int du = -1; du <= 1; ++du) {
                            const int u = t - 1 + du;
                            if(u < 0 || u >= kCol) continue;
                            const int k = k0 + u;
                            const bool ok = okJ && !(exact && (k < max(ck - 1, 0) || k > min(ck + 1, g.G[2] - 1)));
                            const float ddz = (((float)k + 0.5f) * g.dx + g.bmin[2]) - L[w].z;
                            const float d2 = dxy + ddz * ddz;  // glm::length2: (x*x + y*y) + z*z
                            m[uj][u] = fminf(m[uj][u], ok ? d2 : inf);
                        }
                    }
                }
            }
        }
    }
    if(i < g.G[0]) {
#pragma unroll
        for(int uj = 0; uj < kRptSdf; ++uj)
#pragma unroll
            for(int u = 0; u < kCol; ++u) {
                if(j0 + uj >= g.G[1] || k0 + u >= g.G[2]) continue;
                float ph = empty;
                if(m[uj][u] != inf) {
                    const float val = sqrtf(m[uj][u]) - g.sdfRadius;
                    if(val < ph) ph = val;
                }
                phi[cell_index(uj, u)] = ph;
            }
    }
}

static dim3 col_grid(int sx, int sr, int sa, int rpt) {
    return dim3((unsigned)((sx + kLx - 1) / kLx), (unsigned)((sr + kLr * rpt - 1) / (kLr * rpt)),
                (unsigned)((sa + kCol - 1) / kCol));
}

void launch_p2g_col(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                    size_t stride, float* const* out, uint8_t* const* valid, cudaStream_t s) {
    const dim3 blk(kLx, kLr);
    // u, v: rows along y, columns along z; w: rows along z, columns along y
    { k_p2g_col<0><<<col_grid(g.G[0] + 1, g.G[1], g.G[2], kRptP2G), blk, 0, s>>>(g, st, cellStart, rec, stride, out[0], valid[0]); bnn_note_launch(); }
    { k_p2g_col<1><<<col_grid(g.G[0], g.G[1] + 1, g.G[2], kRptP2G), blk, 0, s>>>(g, st, cellStart, rec, stride, out[1], valid[1]); bnn_note_launch(); }
    { k_p2g_col<2><<<col_grid(g.G[0], g.G[2] + 1, g.G[1], kRptP2G), blk, 0, s>>>(g, st, cellStart, rec, stride, out[2], valid[2]); bnn_note_launch(); }
}

void launch_fluid_sdf_col(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                          size_t stride, float* phi, cudaStream_t s) {
    { k_fluid_sdf_col<<<col_grid(g.G[0], g.G[1], g.G[2], kRptSdf), dim3(kLx, kLr), 0, s>>>(g, st, cellStart, rec + 3 * stride,
                                                                               phi); bnn_note_launch(); }
}

} // namespace bnn
