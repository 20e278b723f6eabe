// Matrix-free Jacobi PCG for the 7-point pressure system (PCGSolver::solve_precond,
// BananaCore/Banana/LinearAlgebra/LinearSolvers/PCGSolver.cpp:143-199).
//
// Rows are the fluid cells in linear-cell order.  Per row: diag (float), 1/diag, and six
// neighbour row indices in ascending column order (-z,-y,-x,+x,+y,+z; -1 = none), stored
// as six planes nbr[q*n + r].  With face weights 1 every off-diagonal equals -dt, so the
// matrix is never materialised; with solid boundaries (weights below 1) the off-diagonal
// values ride along: six planes coef[q*n + r] with the compact rows, or two float4 per
// row (k_pack_coef) with the packed ones.
//
// Rows of a grid (rows numbered in cell order) are also packed into one 16-byte record
// each: the x neighbours are always rows r-1 / r+1, so they become two flag bits, the y
// and z neighbours become row distances, and the diagonal rides along.  One load then
// replaces seven, and the x neighbours' values come from the adjacent lanes by warp
// shuffles instead of loads.  Record {y, zm, zp, diag}: y = dy- | dy+ << 16 (row distances
// of the -y / +y neighbours, 0 = none), zm = dz- | (has -x) << 31, zp = dz+ | (has +x) << 31.
//
// The solve is one persistent cooperative kernel; every iteration works in the canonical
// 2048-row chunk layout so the FP64 dot products are bit-reproducible:
//   phase A: s = z + beta*s_old formed on the fly (double buffered), q = A s, partial s.q;
//   grid barrier; every block reduces the partials to the same alpha;
//   phase B: x += alpha s, r -= alpha q, max|r|, z = D^-1 r, partial z.r;
//   grid barrier; every block reduces to the same rho, max|r| and beta.
#include "bnn_internal.cuh"

#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

namespace bnn {

template<class VT> struct Sc;
template<> struct Sc<float> {
    __device__ static float alpha(const DevState* s) { return s->alpha; }
    __device__ static float beta(const DevState* s) { return s->beta; }
    __device__ static void set_alpha(DevState* s, double a) { s->alpha = (float)a; }
    __device__ static void set_beta(DevState* s, double b) { s->beta = (float)b; }
    __device__ static float tol(const DevState* s) { return s->tol; }
    __device__ static void set_tol(DevState* s, float t) { s->tol = t; }
    __device__ static void set_resid(DevState* s, float r) { s->resid = r; s->resid64 = r; }
};
template<> struct Sc<double> {
    __device__ static double alpha(const DevState* s) { return s->alpha64; }
    __device__ static double beta(const DevState* s) { return s->beta64; }
    __device__ static void set_alpha(DevState* s, double a) { s->alpha64 = a; }
    __device__ static void set_beta(DevState* s, double b) { s->beta64 = b; }
    __device__ static double tol(const DevState* s) { return s->tol64; }
    __device__ static void set_tol(DevState* s, double t) { s->tol64 = t; }
    __device__ static void set_resid(DevState* s, double r) { s->resid64 = r; s->resid = (float)r; }
};

template<class VT> __device__ __forceinline__ VT vabs(VT x) { return x < VT(0) ? -x : x; }

template<class VT> __device__ __forceinline__ VT block_max_t(VT v, VT* sm) {
    const int t = threadIdx.x;
    sm[t] = v;
    __syncthreads();
    for(int off = 128; off > 0; off >>= 1) {
        if(t < off) { VT o = sm[t + off]; sm[t] = sm[t] > o ? sm[t] : o; }
        __syncthreads();
    }
    VT r = sm[0];
    __syncthreads();
    return r;
}
template<class VT> __device__ __forceinline__ VT reduce_max_t(const VT* part, int nch, VT* sm) {
    VT acc = VT(0);
    for(int c = threadIdx.x; c < nch; c += kLanes) { VT o = __ldcg(part + c); acc = acc > o ? acc : o; }
    return block_max_t(acc, sm);
}

// ---------------------------------------------------------------------------------
// Persistent PCG: one cooperative launch per solve.  Blocks own fixed 2048-row chunks
// (c = blockIdx.x, +gridDim.x, ...), every phase writes one FP64 partial per chunk, and
// after each grid barrier EVERY block reduces the partials in the canonical order, so all
// blocks hold bit-identical scalars and take the same branch without a broadcast.  Data
// written by other blocks is read with ld.global.cg (L2), never through a stale L1 line.
// ---------------------------------------------------------------------------------
// A barrier wait gives up once it has polled minSpins times and ns more of wall time
// (%globaltimer) have passed, or after maxSpins polls whatever the clock says.  Counting
// polls as well as time keeps a solve that the GPU time-slices away from giving up early.
struct BarrierLimit {
    unsigned long long ns;
    unsigned minSpins, maxSpins;
};
__host__ __device__ constexpr BarrierLimit solve_barrier_limit() { return {1000000000ull, 1u << 20, 1u << 26}; }
// Pause between polls of the barrier word: fewer acquire loads queue at the word's L2
// slice behind the arrivals (1.59M-row solve, us per iteration: 22.59 without a pause,
// 22.42-22.46 at 32 or 100 ns, 22.74 at 256, 22.83-22.92 at 1000; a relaxed poll followed
// by one acquire fence: 23.24)
#ifndef BNN_BARRIER_SLEEP_NS
#define BNN_BARRIER_SLEEP_NS 100
#endif

// Canonical 256-lane tree (lane t of the chunk owns v; levels 128, 64, 32 then a warp
// shuffle tree), with one shared-memory staging step: warp 0 forms the three upper
// levels in registers in the same association as the level-by-level tree.  The sum is
// valid in thread 0.  `m` (optional) is max-reduced alongside.
template<class VT>
__device__ __forceinline__ void block_sum_max_256(double v, VT m, double* sm, VT* smm, double& sum, VT& mx,
                                                  bool withMax) {
    const int t = threadIdx.x;
    sm[t] = v;
    if(withMax) smm[t] = m;
    __syncthreads();
    if(t < 32) {
        const double a0 = sm[t] + sm[t + 128];
        const double a1 = sm[t + 64] + sm[t + 192];
        const double a2 = sm[t + 32] + sm[t + 160];
        const double a3 = sm[t + 96] + sm[t + 224];
        double c = (a0 + a1) + (a2 + a3);
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) c = c + __shfl_down_sync(0xffffffffu, c, off);
        sum = c;
        if(withMax) {
            VT x = smm[t];
#pragma unroll
            for(int q = 1; q < 8; ++q) { const VT o = smm[t + 32 * q]; x = x > o ? x : o; }
#pragma unroll
            for(int off = 16; off > 0; off >>= 1) { const VT o = __shfl_down_sync(0xffffffffu, x, off); x = x > o ? x : o; }
            mx = x;
        }
    }
    __syncthreads();
}

// Reduce the chunk partials (sum in canonical order, and max) and give the result to
// every thread of the block.  A thread's partials (chunks t, t + 256, ...) are loaded four
// at a time before they are added in chunk order; warp 0 forms the block result and lane 0
// publishes it in its own shared slot, so one block barrier separates it from the readers
// (the next write of the slot comes after the next reduction's first barrier, which every
// reader reaches only after reading).
template<class VT>
__device__ __forceinline__ void reduce_partials_bcast(const double* part, const VT* pmax, int nch, double* sm, VT* smm,
                                                      double& sum, VT& mx) {
    __shared__ double sSum;
    __shared__ VT sMax;
    constexpr int U = 4;
    double acc = 0.0;
    VT m = VT(0);
    for(int c0 = threadIdx.x; c0 < nch; c0 += U * kLanes) {
        double p[U];
        VT o[U];
#pragma unroll
        for(int u = 0; u < U; ++u) {
            const int c = c0 + u * kLanes;
            p[u] = c < nch ? __ldcg(part + c) : 0.0;
            o[u] = (pmax && c < nch) ? __ldcg(pmax + c) : VT(0);
        }
#pragma unroll
        for(int u = 0; u < U; ++u)
            if(c0 + u * kLanes < nch) {
                acc = acc + p[u];
                if(pmax) m = m > o[u] ? m : o[u];
            }
    }
    const int t = threadIdx.x;
    sm[t] = acc;
    if(pmax) smm[t] = m;
    __syncthreads();
    if(t < 32) {
        // the association of block_sum_max_256
        const double a0 = sm[t] + sm[t + 128];
        const double a1 = sm[t + 64] + sm[t + 192];
        const double a2 = sm[t + 32] + sm[t + 160];
        const double a3 = sm[t + 96] + sm[t + 224];
        double c = (a0 + a1) + (a2 + a3);
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) c = c + __shfl_down_sync(0xffffffffu, c, off);
        VT x = VT(0);
        if(pmax) {
            x = smm[t];
#pragma unroll
            for(int q = 1; q < 8; ++q) { const VT o = smm[t + 32 * q]; x = x > o ? x : o; }
#pragma unroll
            for(int off = 16; off > 0; off >>= 1) { const VT o = __shfl_down_sync(0xffffffffu, x, off); x = x > o ? x : o; }
        }
        if(t == 0) { sSum = c; sMax = x; }
    }
    __syncthreads();
    sum = sSum;
    mx = sMax;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_add_release_u32(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" : : "l"(p), "r"(v) : "memory");
}

// Grid-wide barrier with a bounded wait (sense reversal on one word, zeroed before the
// launch): block 0 adds 2^31 - (nblocks - 1), every other block adds 1, so the word's top
// bit flips exactly when the last block arrives and its low bits return to where they
// were.  After the b-th barrier the top bit is b & 1; each block counts its barriers in
// `sense`, so the arrival is a fire-and-forget reduction (release) and the poll (acquire)
// starts at once.  Each block's writes before the barrier are visible to every block
// after it.  Returns false (and sets the timeout flag) when the wait gave up.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned nblocks, unsigned& sense, unsigned* flags,
                                             BarrierLimit lim) {
    __shared__ int sOk;
    sense ^= 1u;
    __syncthreads();
    if(threadIdx.x == 0) {
        int ok = 1;
        const unsigned add = blockIdx.x == 0 ? 0x80000000u - (nblocks - 1u) : 1u;
        red_add_release_u32(&gs->count, add);
        unsigned spins = 0;
        unsigned long long t0 = 0;
        while((ld_acquire_u32(&gs->count) >> 31) != sense) {
            ++spins;
            if(spins == lim.minSpins) t0 = global_ns();
            if(spins >= lim.maxSpins || (spins > lim.minSpins && (spins & 255u) == 0u && global_ns() - t0 >= lim.ns)) {
                ok = 0;
                atomicOr(flags, BNN_FLAG_TIMEOUT);
                break;
            }
            if(BNN_BARRIER_SLEEP_NS) __nanosleep(BNN_BARRIER_SLEEP_NS);
        }
        sOk = ok;
    }
    __syncthreads();
    return sOk != 0;
}

template<class VT> struct PcgArgs {
    int n;
    const float* rhsF;
    const float* diag;
    const VT* invd;
    const int32_t* nbr;
    const int4* rec;
    const float* coef;  // compact rows: off-diagonal planes (nullptr: all negoff)
    const float4* coefRow;  // packed rows with coefficients: 2 float4 per row (6 used)
    VT negoff;
    VT tolFactor;
    unsigned maxIter;
    VT *x, *r, *z, *s0, *s1, *q;
    double *part0, *part1, *part2;
    VT* partMax;
    DevState* st;
    GridSync* gs;
};

template<class VT>
__device__ __forceinline__ VT s_val(const VT* z, const VT* sOld, VT beta, bool first, size_t e) {
    return first ? __ldcg(z + e) : __ldcg(z + e) + beta * __ldcg(sOld + e);
}

// Resident blocks per SM the register budget is sized for, and rows per lane whose loads
// are in flight together in the SpMV phase (a divisor of kPerLane).  With the chunk's row
// records loaded before its neighbour loads, three blocks of two rows run best for every
// vector type (1.59M rows, us per iteration: FP32 22.9 against 23.5 at two blocks of four
// rows and 23.9 at two blocks of two; FP64 42.1 against 44.5 and 46.8; rows with
// off-diagonal values 38.5 against 42.6 at two blocks of four rows, which spill).
#ifndef BNN_PCG_MIN_BLOCKS
#define BNN_PCG_MIN_BLOCKS 3
#endif
#ifndef BNN_PCG_ROW_GROUP
#define BNN_PCG_ROW_GROUP 2
#endif
#ifndef BNN_PCG_MIN_BLOCKS_F64
#define BNN_PCG_MIN_BLOCKS_F64 3
#endif
#ifndef BNN_PCG_ROW_GROUP_F64
#define BNN_PCG_ROW_GROUP_F64 2
#endif
#ifndef BNN_PCG_MIN_BLOCKS_COEF
#define BNN_PCG_MIN_BLOCKS_COEF 3
#endif
#ifndef BNN_PCG_ROW_GROUP_COEF
#define BNN_PCG_ROW_GROUP_COEF 2
#endif
template<class VT, bool COEF> constexpr int pcg_min_blocks() {
    return sizeof(VT) == 8 ? BNN_PCG_MIN_BLOCKS_F64 : (COEF ? BNN_PCG_MIN_BLOCKS_COEF : BNN_PCG_MIN_BLOCKS);
}
template<class VT, bool COEF> constexpr int pcg_row_group() {
    return sizeof(VT) == 8 ? BNN_PCG_ROW_GROUP_F64 : (COEF ? BNN_PCG_ROW_GROUP_COEF : BNN_PCG_ROW_GROUP);
}
template<class VT, bool PACKED, bool COEF = false>
__global__ void __launch_bounds__(kLanes, pcg_min_blocks<VT, COEF>()) k_pcg_persistent(PcgArgs<VT> a) {
    constexpr int kRowGroup = pcg_row_group<VT, COEF>();
    static_assert(kPerLane % kRowGroup == 0, "row groups must tile a lane's rows");
    __shared__ double smd[kLanes];
    __shared__ VT smv[kLanes];
    const int n = a.n;
    const int nch = (n + kChunk - 1) / kChunk;
    const unsigned nb = gridDim.x;
    unsigned sense = 0;  // barriers passed, mod 2
    unsigned* flags = &a.st->flags;
    VT* __restrict__ xR = a.x;
    VT* __restrict__ rR = a.r;
    VT* __restrict__ zR = a.z;
    VT* __restrict__ qR = a.q;
    const VT* __restrict__ invdR = a.invd;
    const float* __restrict__ diagR = a.diag;
    const int32_t* __restrict__ nbrR = a.nbr;
    const int4* __restrict__ recR = a.rec;
    const float* __restrict__ coefR = a.coef;
    const VT negoff = a.negoff;
    const int lane = threadIdx.x & 31;

    // ---- init: r = rhs, x = 0, z = D^-1 r; partial z.r and max|r| (PCGSolver.cpp:151-168)
    for(int c = blockIdx.x; c < nch; c += nb) {
        double acc = 0.0;
        VT m = VT(0);
        const size_t base = (size_t)c * kChunk + threadIdx.x;
#pragma unroll
        for(int j = 0; j < kPerLane; ++j) {
            const size_t e = base + (size_t)j * kLanes;
            if(e < (size_t)n) {
                const VT rv = (VT)a.rhsF[e];
                a.r[e] = rv;
                a.x[e] = VT(0);
                const VT ab = vabs(rv);
                m = m > ab ? m : ab;
                const VT zv = __ldg(a.invd + e) * rv;
                a.z[e] = zv;
                acc = acc + (double)zv * (double)rv;
            }
        }
        double bs;
        VT bm;
        block_sum_max_256<VT>(acc, m, smd, smv, bs, bm, true);
        if(threadIdx.x == 0) { a.part0[c] = bs; a.partMax[c] = bm; }
    }
    if(!grid_barrier(a.gs, nb, sense, flags, solve_barrier_limit())) return;
    double rho;
    VT resid;
    reduce_partials_bcast<VT>(a.part0, a.partMax, nch, smd, smv, rho, resid);
    const VT tolFactor = fmax(a.tolFactor, VT(1e-30));
    unsigned iter = 0, success = 0;
    bool done = false;
    VT tol = VT(0);
    if(resid < (VT)FLT_MIN) {
        done = true;
        success = 1;
    } else {
        tol = tolFactor * resid;
        if(rho < (double)FLT_MIN || isnan(rho)) done = true;
    }
    if(a.maxIter == 0) done = true;

    VT beta = VT(0);
    bool first = true;
#ifdef BNN_PCG_TIMING
    unsigned long long tc[6] = {0, 0, 0, 0, 0, 0};
    long long t0_ = clock64();
#define TMARK(k) do { long long t1_ = clock64(); tc[k] += (unsigned long long)(t1_ - t0_); t0_ = t1_; } while(0)
#else
#define TMARK(k) do {} while(0)
#endif
    VT* sOld = a.s1;
    VT* sNew = a.s0;
    while(!done) {
        // ---- phase A: s = z + beta s_old, q = A s, partial s.q (PCGSolver.cpp:173-174,192-193)
        // Every load of a chunk is issued before any store (missing neighbours read the
        // row itself and are masked afterwards), so the chunk costs a few L2 round trips
        // instead of one per row and neighbour.
        for(int c = blockIdx.x; c < nch; c += nb) {
            const size_t base = (size_t)c * kChunk + threadIdx.x;
            VT sOut[kPerLane], qOut[kPerLane];
            // the row records of the whole chunk first: one round trip for all of them
            int4 recAll[PACKED ? kPerLane : 1];
            if constexpr(PACKED) {
#pragma unroll
                for(int j = 0; j < kPerLane; ++j) {
                    const size_t e = base + (size_t)j * kLanes;
                    recAll[j] = __ldg(recR + (e < (size_t)n ? e : 0));
                }
            }
#pragma unroll
            for(int g0 = 0; g0 < kPerLane; g0 += kRowGroup) {
                int32_t id[kRowGroup][7];
                bool has[kRowGroup][7];
                float dg[kRowGroup];
                size_t rowE[kRowGroup];
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
                    const size_t e = base + (size_t)(g0 + u) * kLanes;
                    const size_t ee = e < (size_t)n ? e : 0;
                    if constexpr(PACKED) {
                        // a row past n reads row 0, whose neighbours are all valid rows
                        const int4 rr = recAll[g0 + u];
                        const int dyM = rr.x & 0xffff, dyP = (int)((unsigned)rr.x >> 16);
                        const int dzM = rr.y & 0x7fffffff, dzP = rr.z & 0x7fffffff;
                        const int32_t r0 = (int32_t)ee;
                        has[u][0] = dzM != 0; id[u][0] = r0 - dzM;
                        has[u][1] = dyM != 0; id[u][1] = r0 - dyM;
                        // x neighbours: lanes 0 / 31 load them, the others take a shuffle
                        has[u][2] = rr.y < 0; id[u][2] = (lane == 0 && rr.y < 0) ? r0 - 1 : r0;
                        has[u][3] = true; id[u][3] = r0;
                        has[u][4] = rr.z < 0; id[u][4] = (lane == 31 && rr.z < 0) ? r0 + 1 : r0;
                        has[u][5] = dyP != 0; id[u][5] = r0 + dyP;
                        has[u][6] = dzP != 0; id[u][6] = r0 + dzP;
                        dg[u] = __int_as_float(rr.w);
                    } else {
#pragma unroll
                        for(int q = 0; q < 6; ++q) {
                            const int32_t v = __ldg(nbrR + (size_t)q * n + ee);
                            const int slot = q < 3 ? q : q + 1;
                            has[u][slot] = v >= 0;
                            id[u][slot] = v >= 0 ? v : (int32_t)ee;
                        }
                        rowE[u] = ee;
                        id[u][3] = (int32_t)ee;
                        has[u][3] = true;
                        dg[u] = __ldg(diagR + ee);
                    }
                }
                VT zv[kRowGroup][7], sv[kRowGroup][7];
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u)
#pragma unroll
                    for(int q = 0; q < 7; ++q) {
                        const bool load = !PACKED || (q != 2 && q != 4) || (q == 2 && lane == 0) || (q == 4 && lane == 31);
                        zv[u][q] = load ? __ldcg(zR + id[u][q]) : VT(0);
                        sv[u][q] = (first || !load) ? VT(0) : __ldcg(sOld + id[u][q]);
                    }
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
                    VT s7[7];
#pragma unroll
                    for(int q = 0; q < 7; ++q) s7[q] = first ? zv[u][q] : zv[u][q] + beta * sv[u][q];
                    if constexpr(PACKED) {
                        // rows e-1 / e+1 belong to the neighbouring lanes of this warp
                        const VT up = __shfl_up_sync(0xffffffffu, s7[3], 1);
                        const VT dn = __shfl_down_sync(0xffffffffu, s7[3], 1);
                        if(lane != 0) s7[2] = up;
                        if(lane != 31) s7[4] = dn;
                    }
                    VT t = VT(0);
                    if constexpr(PACKED && COEF) {
                        // the row's off-diagonals in slot order (-z, -y, -x | +x, +y, +z)
                        const size_t e = base + (size_t)(g0 + u) * kLanes;
                        const size_t ee = e < (size_t)n ? e : 0;
                        const float4 c0 = __ldg(a.coefRow + 2 * ee), c1 = __ldg(a.coefRow + 2 * ee + 1);
                        const VT co[7] = {(VT)c0.x, (VT)c0.y, (VT)c0.z, VT(0), (VT)c0.w, (VT)c1.x, (VT)c1.y};
#pragma unroll
                        for(int q = 0; q < 3; ++q) if(has[u][q]) t += co[q] * s7[q];
                        if(dg[u] != 0.f) t += (VT)dg[u] * s7[3];
#pragma unroll
                        for(int q = 4; q < 7; ++q) if(has[u][q]) t += co[q] * s7[q];
                    } else if constexpr(PACKED) {
#pragma unroll
                        for(int q = 0; q < 3; ++q) if(has[u][q]) t += negoff * s7[q];
                        if(dg[u] != 0.f) t += (VT)dg[u] * s7[3];
#pragma unroll
                        for(int q = 4; q < 7; ++q) if(has[u][q]) t += negoff * s7[q];
                    } else {
                        // off-diagonal of slot q (plane q, or q - 1 above the diagonal)
                        auto cf = [&](int q) {
                            return coefR ? (VT)__ldg(coefR + (size_t)(q < 3 ? q : q - 1) * n + rowE[u]) : negoff;
                        };
#pragma unroll
                        for(int q = 0; q < 3; ++q) if(has[u][q]) t += cf(q) * s7[q];
                        if(dg[u] != 0.f) t += (VT)dg[u] * s7[3];
#pragma unroll
                        for(int q = 4; q < 7; ++q) if(has[u][q]) t += cf(q) * s7[q];
                    }
                    sOut[g0 + u] = s7[3];
                    qOut[g0 + u] = t;
                }
            }
            double acc = 0.0;
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                if(e < (size_t)n) {
                    sNew[e] = sOut[j];
                    qR[e] = qOut[j];
                    acc = acc + (double)sOut[j] * (double)qOut[j];
                }
            }
            double bs;
            VT unused;
            block_sum_max_256<VT>(acc, VT(0), smd, smv, bs, unused, false);
            if(threadIdx.x == 0) a.part1[c] = bs;
        }
        TMARK(0);
        if(!grid_barrier(a.gs, nb, sense, flags, solve_barrier_limit())) return;
        TMARK(1);
        double tmp;
        VT unused2;
        reduce_partials_bcast<VT>(a.part1, (const VT*)nullptr, nch, smd, smv, tmp, unused2);
        if(tmp < (double)FLT_MIN) {
            ++iter;
            success = 1;
            break;
        }
        const VT alpha = (VT)(rho / tmp);
        TMARK(2);
        // ---- phase B: x += alpha s, r -= alpha q, max|r|, z = D^-1 r, partial z.r
        for(int c = blockIdx.x; c < nch; c += nb) {
            const size_t base = (size_t)c * kChunk + threadIdx.x;
            VT xs[kPerLane], ss[kPerLane], rs[kPerLane], qs[kPerLane], is[kPerLane];
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                const size_t ee = e < (size_t)n ? e : 0;
                xs[j] = __ldcg(xR + ee);
                ss[j] = __ldcg(sNew + ee);
                rs[j] = __ldcg(rR + ee);
                qs[j] = __ldcg(qR + ee);
                is[j] = __ldg(invdR + ee);
            }
            double acc = 0.0;
            VT m = VT(0);
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                if(e < (size_t)n) {
                    xR[e] = xs[j] + alpha * ss[j];
                    const VT rv = rs[j] + (-alpha) * qs[j];
                    rR[e] = rv;
                    const VT ab = vabs(rv);
                    m = m > ab ? m : ab;
                    const VT zv = is[j] * rv;
                    zR[e] = zv;
                    acc = acc + (double)zv * (double)rv;
                }
            }
            double bs;
            VT bm;
            block_sum_max_256<VT>(acc, m, smd, smv, bs, bm, true);
            if(threadIdx.x == 0) { a.part2[c] = bs; a.partMax[c] = bm; }
        }
        TMARK(3);
        if(!grid_barrier(a.gs, nb, sense, flags, solve_barrier_limit())) return;
        TMARK(4);
        double rhoNew;
        reduce_partials_bcast<VT>(a.part2, a.partMax, nch, smd, smv, rhoNew, resid);
        TMARK(5);
        ++iter;
        if(resid < tol) {
            success = 1;
            break;
        }
        beta = (VT)(rhoNew / rho);
        rho = rhoNew;
        if(iter >= a.maxIter) {
            if(blockIdx.x == 0 && threadIdx.x == 0) atomicOr(flags, BNN_FLAG_PCG_MAXITER);
            break;
        }
        VT* t = sOld;
        sOld = sNew;
        sNew = t;
        first = false;
    }
#ifdef BNN_PCG_TIMING
    if(threadIdx.x == 0) {
        unsigned smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        printf("blk %d sm %u iters %u  cycles/iter: phaseA %.0f bar1 %.0f red1 %.0f phaseB %.0f bar2 %.0f red2 %.0f\n",
               (int)blockIdx.x, smid, iter, tc[0] / (double)iter, tc[1] / (double)iter, tc[2] / (double)iter,
               tc[3] / (double)iter, tc[4] / (double)iter, tc[5] / (double)iter);
    }
#endif
    if(blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->iter = iter;
        a.st->success = success;
        a.st->done = 1;
        Sc<VT>::set_resid(a.st, resid);
    }
}

// ---------------------------------------------------------------------------------
// Single-reduction PCG (Chronopoulos & Gear, 1989): the same Krylov iterates as
// PCGSolver::solve_precond (PCGSolver.cpp:143-199) in exact arithmetic, with both inner
// products of an iteration formed in one reduction, so one grid barrier per iteration
// instead of two.  With u = D^-1 r and w = A u:
//   gamma_i = (r_i, u_i), delta_i = (w_i, u_i)
//   beta_i  = gamma_i / gamma_{i-1},  alpha_i = gamma_i / (delta_i - beta_i gamma_i / alpha_{i-1})
//   p_i = u_i + beta_i p_{i-1},  s_i = w_i + beta_i s_{i-1}   (s_i = A p_i)
//   x_{i+1} = x_i + alpha_i p_i,  r_{i+1} = r_i - alpha_i s_i,  then u_{i+1}, w_{i+1}
// (the denominator is (p_i, A p_i); the first iteration takes beta = 0, alpha = gamma/delta).
// w_{i+1} = A u_{i+1} needs the neighbours' new u.  Instead of a second barrier, a row
// recomputes each neighbour's new u from the neighbour's old record {r, w, s, 1/diag}
// with the exact operations the neighbour uses for itself, so both agree bit for bit.  The
// records are double-buffered (read one, write the other), and so are the chunk partials
// (a block may start the next iteration while another still reads this one's partials).
// Per row and iteration: its own record, p and x, one record per y / z neighbour; the x
// neighbours' u come from the adjacent lanes by shuffles (packed rows).  Scalars are
// formed in FP64 from the canonical FP64 sums and rounded to the vector type.
// ---------------------------------------------------------------------------------
template<class VT> struct alignas(4 * sizeof(VT)) RowState {
    VT r, w, s, inv;
};
template<class VT> __device__ __forceinline__ RowState<VT> ld_state(const RowState<VT>* p) {
    RowState<VT> o;
    if constexpr(sizeof(VT) == 4) {
        const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
        o.r = v.x; o.w = v.y; o.s = v.z; o.inv = v.w;
    } else {
        const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
        o.r = a.x; o.w = a.y; o.s = b.x; o.inv = b.y;
    }
    return o;
}
template<class VT> __device__ __forceinline__ void st_state(RowState<VT>* p, VT r, VT w, VT s, VT inv) {
    if constexpr(sizeof(VT) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(r, w, s, inv);
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2(r, w);
        reinterpret_cast<double2*>(p)[1] = make_double2(s, inv);
    }
}
// The new preconditioned residual of a row from its old record: the row's own update
// written out (s_i = w_i + beta s_{i-1}, r_{i+1} = r_i - alpha s_i, u_{i+1} = r_{i+1} / diag).
template<class VT> __device__ __forceinline__ VT u_next(const RowState<VT>& o, VT alpha, VT beta, bool first) {
    const VT s = first ? o.w : o.w + beta * o.s;
    const VT r = o.r + (-alpha) * s;
    return o.inv * r;
}

template<class VT> struct Cg1Args {
    int n;
    const float* rhsF;
    const float* diag;
    const VT* invd;
    const int32_t* nbr;
    const int4* rec;
    const float* coef;
    const float4* coefRow;
    VT negoff;
    VT tolFactor;
    unsigned maxIter;
    VT *x, *p;
    RowState<VT>* st[2];
    double* part;  // [set 0/1][gamma, delta][nchCap]
    double* pmax;  // [set 0/1][nchCap]
    int nchCap;
    DevState* dst;
    GridSync* gs;
};

// Two canonical 256-lane sums and a max in one block pass (association of
// block_sum_max_256); valid in thread 0.
__device__ __forceinline__ void block_sum2_max_256(double a, double b, double m, double* sa, double* sb, double* sm,
                                                   double& ra, double& rb, double& rm) {
    const int t = threadIdx.x;
    sa[t] = a; sb[t] = b; sm[t] = m;
    __syncthreads();
    if(t < 32) {
        double c[2];
#pragma unroll
        for(int k = 0; k < 2; ++k) {
            const double* sx = k == 0 ? sa : sb;
            const double a0 = sx[t] + sx[t + 128];
            const double a1 = sx[t + 64] + sx[t + 192];
            const double a2 = sx[t + 32] + sx[t + 160];
            const double a3 = sx[t + 96] + sx[t + 224];
            double v = (a0 + a1) + (a2 + a3);
#pragma unroll
            for(int off = 16; off > 0; off >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, off);
            c[k] = v;
        }
        double x = sm[t];
#pragma unroll
        for(int q = 1; q < 8; ++q) { const double o = sm[t + 32 * q]; x = x > o ? x : o; }
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) { const double o = __shfl_down_sync(0xffffffffu, x, off); x = x > o ? x : o; }
        ra = c[0]; rb = c[1]; rm = x;
    }
    __syncthreads();
}

// The chunk partials of both sums (canonical order) and their max, to every thread.
__device__ __forceinline__ void reduce_partials2_bcast(const double* pa, const double* pb, const double* pm, int nch,
                                                       double* sa, double* sb, double* sm, double& ra, double& rb,
                                                       double& rm) {
    __shared__ double sRes[3];
    constexpr int U = 4;
    double acc0 = 0.0, acc1 = 0.0, m = 0.0;
    for(int c0 = threadIdx.x; c0 < nch; c0 += U * kLanes) {
        double x0[U], x1[U], xm[U];
#pragma unroll
        for(int u = 0; u < U; ++u) {
            const int c = c0 + u * kLanes;
            x0[u] = c < nch ? __ldcg(pa + c) : 0.0;
            x1[u] = c < nch ? __ldcg(pb + c) : 0.0;
            xm[u] = c < nch ? __ldcg(pm + c) : 0.0;
        }
#pragma unroll
        for(int u = 0; u < U; ++u)
            if(c0 + u * kLanes < nch) {
                acc0 = acc0 + x0[u];
                acc1 = acc1 + x1[u];
                m = m > xm[u] ? m : xm[u];
            }
    }
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    block_sum2_max_256(acc0, acc1, m, sa, sb, sm, r0, r1, r2);
    if(threadIdx.x == 0) { sRes[0] = r0; sRes[1] = r1; sRes[2] = r2; }
    __syncthreads();
    ra = sRes[0]; rb = sRes[1]; rm = sRes[2];
    __syncthreads();
}

// Rows whose loads a lane keeps in flight together in the single-reduction kernel (each
// row holds seven 4-value records)
#ifndef BNN_CG1_ROW_GROUP
#define BNN_CG1_ROW_GROUP 1
#endif
#ifndef BNN_CG1_MIN_BLOCKS
#define BNN_CG1_MIN_BLOCKS 3
#endif
#ifndef BNN_CG1_MIN_BLOCKS_F64
#define BNN_CG1_MIN_BLOCKS_F64 2
#endif
template<class VT> constexpr int cg1_row_group() { return sizeof(VT) == 8 ? 1 : BNN_CG1_ROW_GROUP; }
template<class VT> constexpr int cg1_min_blocks() { return sizeof(VT) == 8 ? BNN_CG1_MIN_BLOCKS_F64 : BNN_CG1_MIN_BLOCKS; }

template<class VT, bool PACKED, bool COEF>
__global__ void __launch_bounds__(kLanes, cg1_min_blocks<VT>()) k_pcg_cg1(Cg1Args<VT> a) {
    constexpr int kRowGroup = cg1_row_group<VT>();
    __shared__ double sa[kLanes], sb[kLanes], smx[kLanes];
    const int n = a.n;
    const int nch = (n + kChunk - 1) / kChunk;
    const unsigned nb = gridDim.x;
    unsigned sense = 0;
    unsigned* flags = &a.dst->flags;
    const int lane = threadIdx.x & 31;
    const VT negoff = a.negoff;

    // neighbour rows of row ee in slot order (-z,-y,-x,self,+x,+y,+z); a missing one reads
    // the row itself (masked by has)
    auto neighbours = [&](size_t ee, const int4& rr, int32_t id[7], bool has[7], float& dg) {
        if constexpr(PACKED) {
            const int dyM = rr.x & 0xffff, dyP = (int)((unsigned)rr.x >> 16);
            const int dzM = rr.y & 0x7fffffff, dzP = rr.z & 0x7fffffff;
            const int32_t r0 = (int32_t)ee;
            has[0] = dzM != 0; id[0] = r0 - dzM;
            has[1] = dyM != 0; id[1] = r0 - dyM;
            has[2] = rr.y < 0; id[2] = (lane == 0 && rr.y < 0) ? r0 - 1 : r0;
            has[3] = true; id[3] = r0;
            has[4] = rr.z < 0; id[4] = (lane == 31 && rr.z < 0) ? r0 + 1 : r0;
            has[5] = dyP != 0; id[5] = r0 + dyP;
            has[6] = dzP != 0; id[6] = r0 + dzP;
            dg = __int_as_float(rr.w);
        } else {
#pragma unroll
            for(int q = 0; q < 6; ++q) {
                const int32_t v = __ldg(a.nbr + (size_t)q * n + ee);
                const int slot = q < 3 ? q : q + 1;
                has[slot] = v >= 0;
                id[slot] = v >= 0 ? v : (int32_t)ee;
            }
            id[3] = (int32_t)ee;
            has[3] = true;
            dg = __ldg(a.diag + ee);
        }
    };
    // (A v) of a row from its seven slot values, summed in slot order (FixedSparseMatrix::
    // multiply, SparseMatrix.cpp:222-235: column-sorted)
    auto apply_row = [&](size_t ee, const bool has[7], float dg, const VT v7[7]) {
        VT t = VT(0);
        if constexpr(COEF) {
            VT co[7];
            if constexpr(PACKED) {
                const float4 c0 = __ldg(a.coefRow + 2 * ee), c1 = __ldg(a.coefRow + 2 * ee + 1);
                co[0] = (VT)c0.x; co[1] = (VT)c0.y; co[2] = (VT)c0.z; co[3] = VT(0);
                co[4] = (VT)c0.w; co[5] = (VT)c1.x; co[6] = (VT)c1.y;
            } else {
#pragma unroll
                for(int q = 0; q < 7; ++q) co[q] = q == 3 ? VT(0) : (VT)__ldg(a.coef + (size_t)(q < 3 ? q : q - 1) * n + ee);
            }
#pragma unroll
            for(int q = 0; q < 3; ++q) if(has[q]) t += co[q] * v7[q];
            if(dg != 0.f) t += (VT)dg * v7[3];
#pragma unroll
            for(int q = 4; q < 7; ++q) if(has[q]) t += co[q] * v7[q];
        } else {
#pragma unroll
            for(int q = 0; q < 3; ++q) if(has[q]) t += negoff * v7[q];
            if(dg != 0.f) t += (VT)dg * v7[3];
#pragma unroll
            for(int q = 4; q < 7; ++q) if(has[q]) t += negoff * v7[q];
        }
        return t;
    };

    // ---- init: r = b, x = 0, u = D^-1 b, w = A u; gamma, delta, max|r| (set 0)
    for(int c = blockIdx.x; c < nch; c += nb) {
        const size_t base = (size_t)c * kChunk + threadIdx.x;
        double g = 0.0, d = 0.0, m = 0.0;
#pragma unroll 2
        for(int j = 0; j < kPerLane; ++j) {
            const size_t e = base + (size_t)j * kLanes;
            const size_t ee = e < (size_t)n ? e : 0;
            int32_t id[7];
            bool has[7];
            float dg;
            int4 rr = make_int4(0, 0, 0, 0);
            if constexpr(PACKED) rr = __ldg(a.rec + ee);
            neighbours(ee, rr, id, has, dg);
            VT u7[7];
#pragma unroll
            for(int q = 0; q < 7; ++q) {
                const bool load = !PACKED || (q != 2 && q != 4) || (q == 2 && lane == 0) || (q == 4 && lane == 31);
                u7[q] = load ? __ldg(a.invd + id[q]) * (VT)__ldg(a.rhsF + id[q]) : VT(0);
            }
            if constexpr(PACKED) {
                const VT up = __shfl_up_sync(0xffffffffu, u7[3], 1);
                const VT dn = __shfl_down_sync(0xffffffffu, u7[3], 1);
                if(lane != 0) u7[2] = up;
                if(lane != 31) u7[4] = dn;
            }
            const VT wv = apply_row(ee, has, dg, u7);
            if(e < (size_t)n) {
                const VT rv = (VT)a.rhsF[e];
                a.x[e] = VT(0);
                st_state(a.st[0] + e, rv, wv, VT(0), __ldg(a.invd + e));
                g = g + (double)u7[3] * (double)rv;
                d = d + (double)wv * (double)u7[3];
                const double ab = (double)vabs(rv);
                m = m > ab ? m : ab;
            }
        }
        double bg, bd, bm;
        block_sum2_max_256(g, d, m, sa, sb, smx, bg, bd, bm);
        if(threadIdx.x == 0) { a.part[c] = bg; a.part[(size_t)a.nchCap + c] = bd; a.pmax[c] = bm; }
    }
    if(!grid_barrier(a.gs, nb, sense, flags, solve_barrier_limit())) return;
    double gamma, delta, rmax;
    reduce_partials2_bcast(a.part, a.part + a.nchCap, a.pmax, nch, sa, sb, smx, gamma, delta, rmax);
    VT resid = (VT)rmax;
    const VT tolFactor = fmax(a.tolFactor, VT(1e-30));
    unsigned iter = 0, success = 0;
    bool done = false;
    VT tol = VT(0);
    if(resid < (VT)FLT_MIN) {
        done = true;
        success = 1;
    } else {
        tol = tolFactor * resid;
        if(gamma < (double)FLT_MIN || isnan(gamma)) done = true;
    }
    if(a.maxIter == 0) done = true;
    bool first = true;
    double gammaOld = 0.0, a64Old = 0.0;
    int cur = 0, set = 1;
    while(!done) {
        // alpha_i, beta_i; a denominator (p, A p) below FLT_MIN ends the solve as
        // PCGSolver's (p, s) check does (PCGSolver.cpp:173-176)
        double b64 = 0.0, den = delta;
        if(!first) {
            b64 = gamma / gammaOld;
            den = delta - (b64 * gamma) / a64Old;
        }
        if(den < (double)FLT_MIN) {
            ++iter;
            success = 1;
            break;
        }
        const double a64 = gamma / den;
        const VT alpha = (VT)a64, beta = (VT)b64;
        const RowState<VT>* __restrict__ sIn = a.st[cur];
        RowState<VT>* __restrict__ sOut = a.st[1 - cur];
        double* __restrict__ pg = a.part + (size_t)set * 2 * a.nchCap;
        double* __restrict__ pd = pg + a.nchCap;
        double* __restrict__ pm = a.pmax + (size_t)set * a.nchCap;
        for(int c = blockIdx.x; c < nch; c += nb) {
            const size_t base = (size_t)c * kChunk + threadIdx.x;
            int4 recAll[PACKED ? kPerLane : 1];
            if constexpr(PACKED) {
#pragma unroll
                for(int j = 0; j < kPerLane; ++j) {
                    const size_t e = base + (size_t)j * kLanes;
                    recAll[j] = __ldg(a.rec + (e < (size_t)n ? e : 0));
                }
            }
            double g = 0.0, d = 0.0, m = 0.0;
#pragma unroll
            for(int g0 = 0; g0 < kPerLane; g0 += kRowGroup) {
                int32_t id[kRowGroup][7];
                bool has[kRowGroup][7];
                float dg[kRowGroup];
                size_t rowE[kRowGroup];
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
                    const size_t e = base + (size_t)(g0 + u) * kLanes;
                    rowE[u] = e < (size_t)n ? e : 0;
                    neighbours(rowE[u], PACKED ? recAll[g0 + u] : make_int4(0, 0, 0, 0), id[u], has[u], dg[u]);
                }
                RowState<VT> S[kRowGroup][7];
                VT pOld[kRowGroup], xOld[kRowGroup];
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
#pragma unroll
                    for(int q = 0; q < 7; ++q) {
                        const bool load = !PACKED || (q != 2 && q != 4) || (q == 2 && lane == 0) || (q == 4 && lane == 31);
                        if(load) S[u][q] = ld_state(sIn + id[u][q]);
                        else S[u][q] = RowState<VT>{VT(0), VT(0), VT(0), VT(0)};
                    }
                    pOld[u] = first ? VT(0) : __ldcg(a.p + rowE[u]);
                    xOld[u] = __ldcg(a.x + rowE[u]);
                }
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
                    const RowState<VT>& o = S[u][3];
                    const VT uOld = o.inv * o.r;
                    const VT pNew = first ? uOld : uOld + beta * pOld[u];
                    const VT sNew = first ? o.w : o.w + beta * o.s;
                    const VT xNew = xOld[u] + alpha * pNew;
                    const VT rNew = o.r + (-alpha) * sNew;
                    VT u7[7];
#pragma unroll
                    for(int q = 0; q < 7; ++q) u7[q] = q == 3 ? o.inv * rNew : u_next(S[u][q], alpha, beta, first);
                    if constexpr(PACKED) {
                        const VT up = __shfl_up_sync(0xffffffffu, u7[3], 1);
                        const VT dn = __shfl_down_sync(0xffffffffu, u7[3], 1);
                        if(lane != 0) u7[2] = up;
                        if(lane != 31) u7[4] = dn;
                    }
                    const VT wNew = apply_row(rowE[u], has[u], dg[u], u7);
                    const size_t e = base + (size_t)(g0 + u) * kLanes;
                    if(e < (size_t)n) {
                        st_state(sOut + e, rNew, wNew, sNew, o.inv);
                        a.p[e] = pNew;
                        a.x[e] = xNew;
                        g = g + (double)u7[3] * (double)rNew;
                        d = d + (double)wNew * (double)u7[3];
                        const double ab = (double)vabs(rNew);
                        m = m > ab ? m : ab;
                    }
                }
            }
            double bg, bd, bm;
            block_sum2_max_256(g, d, m, sa, sb, smx, bg, bd, bm);
            if(threadIdx.x == 0) { pg[c] = bg; pd[c] = bd; pm[c] = bm; }
        }
        if(!grid_barrier(a.gs, nb, sense, flags, solve_barrier_limit())) return;
        double gNew, dNew, mNew;
        reduce_partials2_bcast(pg, pd, pm, nch, sa, sb, smx, gNew, dNew, mNew);
        resid = (VT)mNew;
        ++iter;
        if(resid < tol) {
            success = 1;
            break;
        }
        if(iter >= a.maxIter) {
            if(blockIdx.x == 0 && threadIdx.x == 0) atomicOr(flags, BNN_FLAG_PCG_MAXITER);
            break;
        }
        gammaOld = gamma;
        gamma = gNew;
        delta = dNew;
        a64Old = a64;
        cur = 1 - cur;
        set = 1 - set;
        first = false;
    }
    if(blockIdx.x == 0 && threadIdx.x == 0) {
        a.dst->iter = iter;
        a.dst->success = success;
        a.dst->done = 1;
        Sc<VT>::set_resid(a.dst, resid);
    }
}

// ---------------------------------------------------------------------------------
// Batched persistent PCG: the Jacobi systems of many scenes (FP32 vectors, grid rows in
// packed records, face weights 1) in one cooperative launch.  A scene's rows are cut into
// the same 2048-row chunks as in a lone solve, and the chunks of all scenes are numbered
// one after another and striped over the blocks (block b takes chunks b, b + grid, ...),
// so as scenes finish the chunks of those still iterating stay spread over the whole grid
// and every block keeps its share of the remaining work.  After each grid barrier a block
// reduces the partials of each scene it works on, a warp per scene
// (warp_reduce_partials: the canonical order over that scene's chunks alone), so every
// scene gets exactly the scalars, iterates and iteration count of a lone
// k_pcg_persistent solve.  Scenes that have finished skip their chunks; the loop ends, for
// all blocks at the same barrier, when a counter of unfinished scenes (decremented by the
// block owning a scene's first chunk) reads 0 right after the first barrier of an
// iteration -- no scene can finish between the last decrement before that barrier and the
// read.
// Yield: a second counter holds the chunks of the unfinished scenes.  When it has fallen to
// yieldBelow (read at the same point), every block leaves at the end of that iteration and
// the owner of each unfinished scene saves its scalars (iterations, rho, beta, tol, last
// residual) to the scene's DevState; the host launches the unfinished scenes again with
// resume set, spread over the whole grid, and they carry on with exactly the iterates they
// had.  Which of the s buffers is the new one follows from the iteration count (even: s0).
// ---------------------------------------------------------------------------------
constexpr int kBatchSlots = 64;  // scenes a block's chunks may belong to

// reduce_partials_bcast's result (the canonical sum over nch chunk partials and their max)
// formed by one warp: lane t stands for the block's threads t, t + 32, ..., t + 224 (the
// threads of block_sum_max_256's first level that lane t of warp 0 combines), each summing
// its partials t', t' + 256, ... in order, then the same association and shuffle tree.
// The result is valid in lane 0.
__device__ __forceinline__ void warp_reduce_partials(const double* part, const float* pmax, int nch, double& sum,
                                                     float& mx) {
    const int lane = threadIdx.x & 31;
    double acc[8];
    float m[8];
#pragma unroll
    for(int v = 0; v < 8; ++v) {
        acc[v] = 0.0;
        m[v] = 0.f;
        for(int c = lane + 32 * v; c < nch; c += kLanes) {
            acc[v] = acc[v] + __ldcg(part + c);
            if(pmax) {
                const float o = __ldcg(pmax + c);
                m[v] = m[v] > o ? m[v] : o;
            }
        }
    }
    // virtual threads lane + 32 v: level 128 pairs v with v + 4, level 64 v = 0/2 with 4/6 ...
    const double a0 = acc[0] + acc[4];
    const double a1 = acc[2] + acc[6];
    const double a2 = acc[1] + acc[5];
    const double a3 = acc[3] + acc[7];
    double c = (a0 + a1) + (a2 + a3);
#pragma unroll
    for(int off = 16; off > 0; off >>= 1) c = c + __shfl_down_sync(0xffffffffu, c, off);
    float x = 0.f;
    if(pmax) {
        x = m[0];
#pragma unroll
        for(int q = 1; q < 8; ++q) { const float o = m[q]; x = x > o ? x : o; }
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) { const float o = __shfl_down_sync(0xffffffffu, x, off); x = x > o ? x : o; }
    }
    sum = c;
    mx = x;
}
struct BatchPcgScene {
    int n;                     // rows
    int resume;                // carry on from the scalars saved at a yield
    const float* rhsF;
    const float* invd;
    const int4* rec;
    float negoff;              // -(1 * dt)
    float tolFactor;
    unsigned maxIter;
    float *x, *r, *z, *s0, *s1, *q;
    double *part0, *part1, *part2;
    float* partMax;
    DevState* dst;             // iterations, success and residual go here
};
struct BatchPcgArgs {
    const BatchPcgScene* sc;
    const unsigned* cp;        // chunk prefix over scenes (ns + 1)
    int ns;
    unsigned total;            // chunks of all scenes
    unsigned perBlock;         // chunks per block
    GridSync* gs;
    unsigned* remaining;       // unfinished scenes
    unsigned* active;          // chunks of the unfinished scenes
    unsigned yieldBelow;       // leave when active has fallen to this (0: never)
    unsigned* flags;           // BNN_FLAG_TIMEOUT
};

__global__ void __launch_bounds__(kLanes, pcg_min_blocks<float, false>()) k_pcg_batch(BatchPcgArgs a) {
    constexpr int kRowGroup = pcg_row_group<float, false>();
    constexpr int kWarps = kLanes / 32;
    __shared__ double smd[kLanes];
    __shared__ float smv[kLanes];
    __shared__ double sRho[kBatchSlots];
    __shared__ float sTol[kBatchSlots], sResid[kBatchSlots], sAlpha[kBatchSlots], sBeta[kBatchSlots];
    __shared__ unsigned sIter[kBatchSlots];
    // 0 iterating, 1 finished, 2 no solve, 3 finished in this iteration's first half
    // (counted off after the second barrier)
    __shared__ int sState[kBatchSlots];
    __shared__ int sScene[kBatchSlots];
    __shared__ unsigned char sSlotOf[kBatchSlots];  // slot of the block's k-th chunk
    __shared__ int sNslots;
    const unsigned nb = gridDim.x;
    unsigned sense = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // The block's chunks are blockIdx.x + k nb (k < nmine): striped over the grid, so the
    // chunks of the scenes still iterating stay spread over all blocks as others finish.
    // Its slots are the scenes those chunks belong to, in order.
    const unsigned nmine = blockIdx.x < a.total ? (a.total - 1 - blockIdx.x) / nb + 1 : 0u;
    if(nmine > (unsigned)kBatchSlots) {  // the host keeps chunks per block within the slot table
        if(threadIdx.x == 0) atomicOr(a.flags, BNN_FLAG_TIMEOUT);
        return;
    }
    if(threadIdx.x == 0) {
        int m = 0, last = -1;
        for(unsigned k = 0; k < nmine; ++k) {
            const int sc = seg_of(a.cp, a.ns, blockIdx.x + k * nb);
            if(sc != last) { sScene[m++] = sc; last = sc; }
            sSlotOf[k] = (unsigned char)(m - 1);
        }
        sNslots = m;
    }
    __syncthreads();
    const int nslots = sNslots;
    // the block owning a scene's first chunk reports its result and counts it off
    auto owner = [&](int sc) { return __ldg(a.cp + sc) % nb == blockIdx.x; };
    auto count_off = [&](int sc) {
        atomicSub(a.remaining, 1u);
        atomicSub(a.active, __ldg(a.cp + sc + 1) - __ldg(a.cp + sc));
    };
    // one thread: the scene of slot j is done (deferred: counted off after the second barrier)
    auto finish1 = [&](int j, unsigned success, bool deferred) {
        const int sc = sScene[j];
        sState[j] = deferred ? 3 : 1;
        if(owner(sc)) {
            DevState* d = a.sc[sc].dst;
            d->iter = sIter[j];
            d->success = success;
            d->done = 1;
            d->resid = sResid[j];
            d->resid64 = sResid[j];
            if(!deferred) count_off(sc);
        }
    };
    auto chunks_of = [&](int sc) { return (int)(__ldg(a.cp + sc + 1) - __ldg(a.cp + sc)); };

    // ---- init: r = rhs, x = 0, z = D^-1 r; partial z.r and max|r| (not for a resumed scene)
    for(unsigned k = 0; k < nmine; ++k) {
        const unsigned c = blockIdx.x + k * nb;
        const int sc = sScene[sSlotOf[k]];
        const BatchPcgScene& S = a.sc[sc];
        if(S.resume) continue;
        const int n = S.n;
        const unsigned lc = c - __ldg(a.cp + sc);
        double acc = 0.0;
        float m = 0.f;
        const size_t base = (size_t)lc * kChunk + threadIdx.x;
#pragma unroll
        for(int j = 0; j < kPerLane; ++j) {
            const size_t e = base + (size_t)j * kLanes;
            if(e < (size_t)n) {
                const float rv = S.rhsF[e];
                S.r[e] = rv;
                S.x[e] = 0.f;
                const float ab = vabs(rv);
                m = m > ab ? m : ab;
                const float zv = __ldg(S.invd + e) * rv;
                S.z[e] = zv;
                acc = acc + (double)zv * (double)rv;
            }
        }
        double bs;
        float bm;
        block_sum_max_256<float>(acc, m, smd, smv, bs, bm, true);
        if(threadIdx.x == 0) { S.part0[lc] = bs; S.partMax[lc] = bm; }
    }
    if(!grid_barrier(a.gs, nb, sense, a.flags, solve_barrier_limit())) return;
    // the scenes' first scalars, a warp per slot
    for(int j = warp; j < nslots; j += kWarps) {
        const int sc = sScene[j];
        const BatchPcgScene& S = a.sc[sc];
        const int nch = chunks_of(sc);
        if(S.resume) {
            // the scalars saved at the yield
            if(lane == 0) {
                const DevState* d = S.dst;
                sIter[j] = d->iter; sRho[j] = d->rho; sBeta[j] = d->beta; sTol[j] = d->tol; sResid[j] = d->resid;
                sState[j] = 0;
            }
            continue;
        }
        double rho = 0.0;
        float resid = 0.f;
        if(nch > 0) warp_reduce_partials(S.part0, S.partMax, nch, rho, resid);
        if(lane == 0) {
            sIter[j] = 0;
            sState[j] = nch > 0 ? 0 : 2;
            sBeta[j] = 0.f;
            if(nch > 0) {
                sRho[j] = rho;
                sResid[j] = resid;
                const float tolFactor = fmaxf(S.tolFactor, 1e-30f);
                if(resid < FLT_MIN) {
                    finish1(j, 1u, false);
                } else {
                    sTol[j] = tolFactor * resid;
                    if(rho < (double)FLT_MIN || isnan(rho) || S.maxIter == 0) finish1(j, 0u, false);
                }
            }
        }
    }
    __syncthreads();

    // a scene's new s is s0 after an even number of iterations, as the lone solve's swap;
    // its first iteration (no s yet) is the one with 0 iterations done
    for(;;) {
        // ---- phase A: s = z + beta s_old, q = A s, partial s.q
        for(unsigned k = 0; k < nmine; ++k) {
            const int jslot = sSlotOf[k];
            if(sState[jslot] != 0) continue;
            const unsigned c = blockIdx.x + k * nb;
            const int sc = sScene[jslot];
            const BatchPcgScene& S = a.sc[sc];
            const int n = S.n;
            const unsigned lc = c - __ldg(a.cp + sc);
            const float beta = sBeta[jslot];
            const float negoff = S.negoff;
            const float* __restrict__ zR = S.z;
            const bool parity = (sIter[jslot] & 1u) != 0;
            const bool first = sIter[jslot] == 0;
            const float* __restrict__ sOld = parity ? S.s0 : S.s1;
            float* __restrict__ sNew = parity ? S.s1 : S.s0;
            const size_t base = (size_t)lc * kChunk + threadIdx.x;
            float sOut[kPerLane], qOut[kPerLane];
            int4 recAll[kPerLane];
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                recAll[j] = __ldg(S.rec + (e < (size_t)n ? e : 0));
            }
#pragma unroll
            for(int g0 = 0; g0 < kPerLane; g0 += kRowGroup) {
                int32_t id[kRowGroup][7];
                bool has[kRowGroup][7];
                float dg[kRowGroup];
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
                    const size_t e = base + (size_t)(g0 + u) * kLanes;
                    const size_t ee = e < (size_t)n ? e : 0;
                    const int4 rr = recAll[g0 + u];
                    const int dyM = rr.x & 0xffff, dyP = (int)((unsigned)rr.x >> 16);
                    const int dzM = rr.y & 0x7fffffff, dzP = rr.z & 0x7fffffff;
                    const int32_t r0 = (int32_t)ee;
                    has[u][0] = dzM != 0; id[u][0] = r0 - dzM;
                    has[u][1] = dyM != 0; id[u][1] = r0 - dyM;
                    has[u][2] = rr.y < 0; id[u][2] = (lane == 0 && rr.y < 0) ? r0 - 1 : r0;
                    has[u][3] = true; id[u][3] = r0;
                    has[u][4] = rr.z < 0; id[u][4] = (lane == 31 && rr.z < 0) ? r0 + 1 : r0;
                    has[u][5] = dyP != 0; id[u][5] = r0 + dyP;
                    has[u][6] = dzP != 0; id[u][6] = r0 + dzP;
                    dg[u] = __int_as_float(rr.w);
                }
                float zv[kRowGroup][7], sv[kRowGroup][7];
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u)
#pragma unroll
                    for(int q = 0; q < 7; ++q) {
                        const bool load = (q != 2 && q != 4) || (q == 2 && lane == 0) || (q == 4 && lane == 31);
                        zv[u][q] = load ? __ldcg(zR + id[u][q]) : 0.f;
                        sv[u][q] = (first || !load) ? 0.f : __ldcg(sOld + id[u][q]);
                    }
#pragma unroll
                for(int u = 0; u < kRowGroup; ++u) {
                    float s7[7];
#pragma unroll
                    for(int q = 0; q < 7; ++q) s7[q] = first ? zv[u][q] : zv[u][q] + beta * sv[u][q];
                    const float up = __shfl_up_sync(0xffffffffu, s7[3], 1);
                    const float dn = __shfl_down_sync(0xffffffffu, s7[3], 1);
                    if(lane != 0) s7[2] = up;
                    if(lane != 31) s7[4] = dn;
                    float t = 0.f;
#pragma unroll
                    for(int q = 0; q < 3; ++q) if(has[u][q]) t += negoff * s7[q];
                    if(dg[u] != 0.f) t += dg[u] * s7[3];
#pragma unroll
                    for(int q = 4; q < 7; ++q) if(has[u][q]) t += negoff * s7[q];
                    sOut[g0 + u] = s7[3];
                    qOut[g0 + u] = t;
                }
            }
            double acc = 0.0;
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                if(e < (size_t)n) {
                    sNew[e] = sOut[j];
                    S.q[e] = qOut[j];
                    acc = acc + (double)sOut[j] * (double)qOut[j];
                }
            }
            double bs;
            float unused;
            block_sum_max_256<float>(acc, 0.f, smd, smv, bs, unused, false);
            if(threadIdx.x == 0) S.part1[lc] = bs;
        }
        if(!grid_barrier(a.gs, nb, sense, a.flags, solve_barrier_limit())) return;
        if(ld_acquire_u32(a.remaining) == 0u) break;
        const bool yieldNow = a.yieldBelow != 0u && ld_acquire_u32(a.active) <= a.yieldBelow;
        // alpha of every scene this block works on, a warp per slot
        for(int j = warp; j < nslots; j += kWarps) {
            if(sState[j] != 0) continue;
            const int sc = sScene[j];
            double tmp;
            float unused2;
            warp_reduce_partials(a.sc[sc].part1, nullptr, chunks_of(sc), tmp, unused2);
            if(lane == 0) {
                if(tmp < (double)FLT_MIN) {
                    ++sIter[j];
                    finish1(j, 1u, true);
                } else {
                    sAlpha[j] = (float)(sRho[j] / tmp);
                }
            }
        }
        __syncthreads();
        // ---- phase B: x += alpha s, r -= alpha q, max|r|, z = D^-1 r, partial z.r
        for(unsigned k = 0; k < nmine; ++k) {
            const int jslot = sSlotOf[k];
            if(sState[jslot] != 0) continue;
            const unsigned c = blockIdx.x + k * nb;
            const int sc = sScene[jslot];
            const BatchPcgScene& S = a.sc[sc];
            const int n = S.n;
            const unsigned lc = c - __ldg(a.cp + sc);
            const float alpha = sAlpha[jslot];
            const float* __restrict__ sNew = (sIter[jslot] & 1u) ? S.s1 : S.s0;
            const size_t base = (size_t)lc * kChunk + threadIdx.x;
            float xs[kPerLane], ss[kPerLane], rs[kPerLane], qs[kPerLane], is[kPerLane];
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                const size_t ee = e < (size_t)n ? e : 0;
                xs[j] = __ldcg(S.x + ee);
                ss[j] = __ldcg(sNew + ee);
                rs[j] = __ldcg(S.r + ee);
                qs[j] = __ldcg(S.q + ee);
                is[j] = __ldg(S.invd + ee);
            }
            double acc = 0.0;
            float m = 0.f;
#pragma unroll
            for(int j = 0; j < kPerLane; ++j) {
                const size_t e = base + (size_t)j * kLanes;
                if(e < (size_t)n) {
                    S.x[e] = xs[j] + alpha * ss[j];
                    const float rv = rs[j] + (-alpha) * qs[j];
                    S.r[e] = rv;
                    const float ab = vabs(rv);
                    m = m > ab ? m : ab;
                    const float zv = is[j] * rv;
                    S.z[e] = zv;
                    acc = acc + (double)zv * (double)rv;
                }
            }
            double bs;
            float bm;
            block_sum_max_256<float>(acc, m, smd, smv, bs, bm, true);
            if(threadIdx.x == 0) { S.part2[lc] = bs; S.partMax[lc] = bm; }
        }
        if(!grid_barrier(a.gs, nb, sense, a.flags, solve_barrier_limit())) return;
        for(int j = warp; j < nslots; j += kWarps) {
            if(sState[j] == 3) {
                if(lane == 0) {
                    if(owner(sScene[j])) count_off(sScene[j]);
                    sState[j] = 1;
                }
                continue;
            }
            if(sState[j] != 0) continue;
            const int sc = sScene[j];
            const BatchPcgScene& S = a.sc[sc];
            double rhoNew;
            float resid;
            warp_reduce_partials(S.part2, S.partMax, chunks_of(sc), rhoNew, resid);
            if(lane == 0) {
                ++sIter[j];
                sResid[j] = resid;
                if(resid < sTol[j]) {
                    finish1(j, 1u, false);
                } else {
                    sBeta[j] = (float)(rhoNew / sRho[j]);
                    sRho[j] = rhoNew;
                    if(sIter[j] >= S.maxIter) {
                        if(owner(sc)) atomicOr(&S.dst->flags, BNN_FLAG_PCG_MAXITER);
                        finish1(j, 0u, false);
                    }
                }
            }
        }
        __syncthreads();
        if(yieldNow) {
            // every block leaves here; each unfinished scene's owner saves its scalars
            for(int j = 0; j < nslots; ++j) {
                const int sc = sScene[j];
                if(sState[j] != 0 || threadIdx.x != 0 || !owner(sc)) continue;
                DevState* d = a.sc[sc].dst;
                d->iter = sIter[j]; d->rho = sRho[j]; d->beta = sBeta[j]; d->tol = sTol[j]; d->resid = sResid[j];
                d->done = 0;
            }
            return;
        }
    }
}

// ---- iterative refinement helpers -------------------------------------------------
// Last-block-done over a block's share `blk` of a launch (the batched launches give every
// scene its own share, so the count to reach is the share's, not gridDim.x)
__device__ __forceinline__ bool last_block_of(unsigned* counter, unsigned nblocks) {
    __shared__ bool amLast;
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0) amLast = atomicAdd(counter, 1u) == nblocks - 1;
    __syncthreads();
    return amLast;
}
// x64 = 0, r64 = b, outer_bmax = outer_res = max|b|
__device__ __forceinline__ void ir_init_body(Blk blk, int n, const float* __restrict__ b, double* __restrict__ x64,
                                             double* __restrict__ r64, double* __restrict__ partMax, DevState* st) {
    __shared__ double sm[kLanes];
    const size_t base = (size_t)blk.x * kChunk + threadIdx.x;
    double m = 0.0;
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            const double bv = (double)b[e];
            x64[e] = 0.0;
            r64[e] = bv;
            const double a = vabs(bv);
            m = m > a ? m : a;
        }
    }
    const double bm = block_max_t(m, sm);
    if(threadIdx.x == 0) partMax[blk.x] = bm;
    if(last_block_of(&st->counter3, blk.n)) {
        const double mx = reduce_max_t(partMax, (int)blk.n, sm);
        if(threadIdx.x == 0) { st->counter3 = 0; st->outer_bmax = mx; st->outer_res = mx; }
    }
}
__global__ void __launch_bounds__(kLanes) k_ir_init(int n, const float* __restrict__ b, double* __restrict__ x64,
                                                    double* __restrict__ r64, double* __restrict__ partMax,
                                                    DevState* st) {
    ir_init_body(own_blk(), n, b, x64, r64, partMax, st);
}
// r32 = (float) r64
__global__ void k_ir_to_f32(int n, const double* __restrict__ r64, float* __restrict__ r32) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) r32[e] = (float)r64[e];
}
__global__ void k_ir_accumulate(int n, double* __restrict__ x64, const float* __restrict__ d) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) x64[e] = x64[e] + (double)d[e];
}
// r64 = b - A x64 in FP64, outer_res = max|r64|
__device__ __forceinline__ void ir_residual_body(Blk blk, int n, const float* __restrict__ b,
                                                 const double* __restrict__ x64, double* __restrict__ r64,
                                                 const float* __restrict__ diag, const int32_t* __restrict__ nbr,
                                                 const float* __restrict__ coef, double negoff,
                                                 double* __restrict__ partMax, DevState* st) {
    __shared__ double sm[kLanes];
    const size_t base = (size_t)blk.x * kChunk + threadIdx.x;
    double m = 0.0;
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            const int32_t nn[6] = {nbr[e], nbr[(size_t)n + e], nbr[2 * (size_t)n + e], nbr[3 * (size_t)n + e],
                                   nbr[4 * (size_t)n + e], nbr[5 * (size_t)n + e]};
            double co[6];
#pragma unroll
            for(int q = 0; q < 6; ++q) co[q] = coef ? (double)coef[(size_t)q * n + e] : negoff;
            double t = 0.0;
            if(nn[0] >= 0) t += co[0] * x64[nn[0]];
            if(nn[1] >= 0) t += co[1] * x64[nn[1]];
            if(nn[2] >= 0) t += co[2] * x64[nn[2]];
            if(diag[e] != 0.f) t += (double)diag[e] * x64[e];
            if(nn[3] >= 0) t += co[3] * x64[nn[3]];
            if(nn[4] >= 0) t += co[4] * x64[nn[4]];
            if(nn[5] >= 0) t += co[5] * x64[nn[5]];
            const double rv = (double)b[e] - t;
            r64[e] = rv;
            const double a = vabs(rv);
            m = m > a ? m : a;
        }
    }
    const double bm = block_max_t(m, sm);
    if(threadIdx.x == 0) partMax[blk.x] = bm;
    if(last_block_of(&st->counter3, blk.n)) {
        const double mx = reduce_max_t(partMax, (int)blk.n, sm);
        if(threadIdx.x == 0) { st->counter3 = 0; st->outer_res = mx; }
    }
}
__global__ void __launch_bounds__(kLanes) k_ir_residual(int n, const float* __restrict__ b,
                                                        const double* __restrict__ x64, double* __restrict__ r64,
                                                        const float* __restrict__ diag,
                                                        const int32_t* __restrict__ nbr,
                                                        const float* __restrict__ coef, double negoff,
                                                        double* __restrict__ partMax, DevState* st) {
    ir_residual_body(own_blk(), n, b, x64, r64, diag, nbr, coef, negoff, partMax, st);
}
__global__ void k_inv_diag64(int n, const float* __restrict__ diag, double* __restrict__ inv) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) inv[e] = diag[e] != 0.f ? 1.0 / (double)diag[e] : 0.0;
}
__global__ void k_f32_to_f64(int n, const float* __restrict__ a, double* __restrict__ b) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) b[e] = (double)a[e];
}
__global__ void k_d64_to_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) b[e] = (float)a[e];
}

// Packs rows of a grid into the 16-byte records (layout at the top of this file).  The
// caller guarantees the x neighbours are rows r-1 / r+1 and the y distances fit 16 bits.
__global__ void k_pack_rows(int n, const float* __restrict__ diag, const int32_t* __restrict__ nbr,
                            int4* __restrict__ rec) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= n) return;
    int32_t nb[6];
#pragma unroll
    for(int q = 0; q < 6; ++q) nb[q] = nbr[(size_t)q * n + r];
    const unsigned dyM = nb[1] >= 0 ? (unsigned)(r - nb[1]) : 0u, dyP = nb[4] >= 0 ? (unsigned)(nb[4] - r) : 0u;
    const unsigned dzM = nb[0] >= 0 ? (unsigned)(r - nb[0]) : 0u, dzP = nb[5] >= 0 ? (unsigned)(nb[5] - r) : 0u;
    int4 v;
    v.x = (int)(dyM | (dyP << 16));
    v.y = (int)(dzM | (nb[2] >= 0 ? 0x80000000u : 0u));
    v.z = (int)(dzP | (nb[3] >= 0 ? 0x80000000u : 0u));
    v.w = __float_as_int(diag[r]);
    rec[r] = v;
}
// The off-diagonal planes of the rows as 2 float4 per row (6 values, plane order)
__global__ void k_pack_coef(int n, const float* __restrict__ coef, float4* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= n) return;
    float c[6];
#pragma unroll
    for(int q = 0; q < 6; ++q) c[q] = coef[(size_t)q * n + r];
    out[2 * (size_t)r] = make_float4(c[0], c[1], c[2], c[3]);
    out[2 * (size_t)r + 1] = make_float4(c[4], c[5], 0.f, 0.f);
}

// ---------------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------------

// Process-wide record of the cooperative PCG kernels: SM count, resident blocks per SM of
// each variant, and the share of the GPU held by solves in flight.  A share is counted
// in units of 1/840 SM (840 is divisible by every resident-block count 1..8).
constexpr int kShareUnits = 840;
struct CoopState {
    std::mutex mu;
    std::condition_variable cv;
    int numSM = 0;
    int perSM[16] = {};
    long long held = 0;
};
static CoopState g_coop;

// Holds `units` of the GPU for the lifetime of the object; waits while other solves hold
// so much that this grid would not fit beside them.
struct CoopShare {
    long long units;
    CoopShare(long long u, long long capacity) : units(u < capacity ? u : capacity) {
        std::unique_lock<std::mutex> lk(g_coop.mu);
        g_coop.cv.wait(lk, [&] { return g_coop.held + units <= capacity; });
        g_coop.held += units;
    }
    ~CoopShare() {
        {
            std::lock_guard<std::mutex> lk(g_coop.mu);
            g_coop.held -= units;
        }
        g_coop.cv.notify_all();
    }
};

int pcg_reserve(PcgWork& w, int n, bool fp64) {
    if(n <= w.cap && (!fp64 || w.x64)) return BNN_OK;
    if(n > w.cap) {
        pcg_release(w);
        const int cap = (int)(n * 1.25) + 4096;
        const size_t nch = ((size_t)cap + kChunk - 1) / kChunk + 1;
        w.nchCap = (int)nch;
        BNN_CUDA_CHECK(dev_alloc(&w.x, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.r, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.z, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.s0, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.s1, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.q, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.d32, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.r32, cap * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.rec, cap * sizeof(int4)));
        BNN_CUDA_CHECK(dev_alloc(&w.part, 3 * nch * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.gs, sizeof(GridSync)));
        BNN_CUDA_CHECK(cudaMemset(w.gs, 0, sizeof(GridSync)));
        BNN_CUDA_CHECK(dev_alloc(&w.partMaxF, nch * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&w.partMaxD, nch * sizeof(double)));
        w.cap = cap;
    }
    for(auto& e : w.ev)
        if(!e) BNN_CUDA_CHECK(cudaEventCreate(&e));
    if(!w.st32[0]) {
        // single-reduction solve: double-buffered row records and partials
        for(int b = 0; b < 2; ++b) BNN_CUDA_CHECK(dev_alloc(&w.st32[b], w.cap * sizeof(float4)));
        BNN_CUDA_CHECK(dev_alloc(&w.cgPart, 4 * (size_t)w.nchCap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.cgMax, 2 * (size_t)w.nchCap * sizeof(double)));
    }
    if(fp64 && !w.st64[0])
        for(int b = 0; b < 2; ++b) BNN_CUDA_CHECK(dev_alloc(&w.st64[b], w.cap * 4 * sizeof(double)));
    if(fp64 && !w.x64) {
        BNN_CUDA_CHECK(dev_alloc(&w.x64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.r64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.z64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.s064, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.s164, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.q64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(dev_alloc(&w.inv64, w.cap * sizeof(double)));
    }
    return BNN_OK;
}

void pcg_release(PcgWork& w) {
    for(auto& e : w.ev)
        if(e) cudaEventDestroy(e);
    for(void* p : {(void*)w.rec, (void*)w.coefRow, (void*)w.x, (void*)w.r, (void*)w.z, (void*)w.s0, (void*)w.s1, (void*)w.q, (void*)w.d32, (void*)w.r32,
                   (void*)w.part, (void*)w.partMaxF, (void*)w.partMaxD, (void*)w.x64, (void*)w.r64, (void*)w.z64,
                   (void*)w.s064, (void*)w.s164, (void*)w.q64, (void*)w.inv64, (void*)w.gs, (void*)w.st32[0],
                   (void*)w.st32[1], (void*)w.st64[0], (void*)w.st64[1], (void*)w.cgPart, (void*)w.cgMax})
        if(p) dev_free(p);
    w = PcgWork();
}

// Runs one PCG solve (VT vectors) as a single cooperative launch.  Returns BNN status;
// the solution is left in x.
template<class VT>
static int pcg_solve_t(PcgWork& w, int n, const float* rhsF, const float* diag, const VT* invd, const int32_t* nbr,
                       const int4* rec, const float* coef, const float4* coefRow, VT negoff, VT tolFactor, unsigned maxIter, VT* x, VT* r, VT* z, VT* s0, VT* s1, VT* q,
                       VT* partMax, bool twoReductions, DevState* dst, DevState* hst, cudaStream_t s, PcgOutcome& out) {
    out = PcgOutcome();
    if(n == 0) { out.success = 1; return BNN_OK; }
    const int nch = (n + kChunk - 1) / kChunk;
    const bool packedCoef = rec && coefRow;
    // kernel variant: bit 0 FP64, bit 1 packed rows, bit 2 coefficients, bit 3 single reduction
    const int ti = (sizeof(VT) == 8 ? 1 : 0) + (rec ? 2 : 0) + ((coef || coefRow) ? 4 : 0) + (twoReductions ? 0 : 8);
    const void* kern;
    if(twoReductions)
        kern = packedCoef ? (const void*)k_pcg_persistent<VT, true, true>
                          : (rec ? (const void*)k_pcg_persistent<VT, true> : (const void*)k_pcg_persistent<VT, false>);
    else if(rec)
        kern = coefRow ? (const void*)k_pcg_cg1<VT, true, true> : (const void*)k_pcg_cg1<VT, true, false>;
    else
        kern = coef ? (const void*)k_pcg_cg1<VT, false, true> : (const void*)k_pcg_cg1<VT, false, false>;
    int numSM = 0, perSMv = 0;
    {
        std::lock_guard<std::mutex> lk(g_coop.mu);
        if(!g_coop.numSM) {
            int dev = 0;
            BNN_CUDA_CHECK(cudaGetDevice(&dev));
            BNN_CUDA_CHECK(cudaDeviceGetAttribute(&g_coop.numSM, cudaDevAttrMultiProcessorCount, dev));
        }
        if(!g_coop.perSM[ti]) {
            BNN_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_coop.perSM[ti], kern, kLanes, 0));
            if(g_coop.perSM[ti] < 1) { bnn_set_error("persistent PCG kernel cannot be resident"); return BNN_ERR_CUDA; }
        }
        numSM = g_coop.numSM;
        perSMv = g_coop.perSM[ti];
    }
    const int cap = numSM * perSMv;
    const int perBlock = (nch + cap - 1) / cap;           // chunks per block
    const int grid = (nch + perBlock - 1) / perBlock;     // balanced: every block the same count
    PcgArgs<VT> a;
    a.n = n; a.rhsF = rhsF; a.diag = diag; a.invd = invd; a.nbr = nbr; a.rec = rec; a.coef = coef; a.coefRow = coefRow; a.negoff = negoff; a.tolFactor = tolFactor;
    a.maxIter = maxIter; a.x = x; a.r = r; a.z = z; a.s0 = s0; a.s1 = s1; a.q = q;
    a.part0 = w.part; a.part1 = w.part + w.nchCap; a.part2 = w.part + 2 * (size_t)w.nchCap; a.partMax = partMax;
    a.st = dst; a.gs = w.gs;
    Cg1Args<VT> c;
    c.n = n; c.rhsF = rhsF; c.diag = diag; c.invd = invd; c.nbr = nbr; c.rec = rec; c.coef = coef; c.coefRow = coefRow;
    c.negoff = negoff; c.tolFactor = tolFactor; c.maxIter = maxIter; c.x = x; c.p = s0;
    for(int b = 0; b < 2; ++b)
        c.st[b] = sizeof(VT) == 8 ? (RowState<VT>*)(void*)w.st64[b] : (RowState<VT>*)(void*)w.st32[b];
    c.part = w.cgPart; c.pmax = w.cgMax; c.nchCap = w.nchCap; c.dst = dst; c.gs = w.gs;
    BNN_CUDA_CHECK(cudaMemsetAsync(&w.gs->count, 0, sizeof(unsigned), s));
    void* args[] = {twoReductions ? (void*)&a : (void*)&c};
    // grids of concurrent solves (several solver handles on several host threads) must
    // fit the GPU together, or blocks of one could wait for SMs held by another's barrier
    CoopShare share(grid * (kShareUnits / perSMv), numSM * kShareUnits);
    if(w.ev[0]) BNN_CUDA_CHECK(cudaEventRecord(w.ev[0], s));
    BNN_CUDA_CHECK(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kLanes), args, 0, s));
    bnn_note_launch();
    if(w.ev[1]) BNN_CUDA_CHECK(cudaEventRecord(w.ev[1], s));
    BNN_CUDA_CHECK(cudaMemcpyAsync(hst, dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    if(w.ev[0] && w.ev[1]) {
        float ms = 0.f;
        if(cudaEventElapsedTime(&ms, w.ev[0], w.ev[1]) == cudaSuccess) out.kernelMs = ms;
    }
    if(hst->flags & BNN_FLAG_TIMEOUT) { bnn_set_error("PCG grid barrier timed out"); return BNN_ERR_TIMEOUT; }
    out.iterations = hst->iter;
    out.success = hst->success;
    out.residual = sizeof(VT) == 8 ? hst->resid64 : (double)hst->resid;
    return BNN_OK;
}

// mode: BNN_PCG_FP32 / FP64 / REFINED, optionally with BNN_PCG_SINGLE_REDUCTION.  Pressure
// written to `pressure` (float, n).
int pcg_solve(PcgWork& w, int n, const float* rhs, const float* diag, const float* invd, const int32_t* nbr,
              const float* coef, bool gridRows, float dt, int modeFlags, float tol, unsigned maxIter, float innerTol,
              float outerTol, float* pressure, double* x64out, DevState* dst, DevState* hst, cudaStream_t s,
              PcgOutcome& out) {
    const int mode = modeFlags & BNN_PCG_MODE_MASK;
    const bool two = (modeFlags & BNN_PCG_SINGLE_REDUCTION) == 0;
    int rc = pcg_reserve(w, n, mode != BNN_PCG_FP32);
    if(rc != BNN_OK) return rc;
    const unsigned nb = (unsigned)((n + 255) / 256);
    const unsigned nch = (unsigned)((n + kChunk - 1) / kChunk);
    out = PcgOutcome();
    const int4* rec = nullptr;
    const float4* coefRow = nullptr;
    if(gridRows && n > 0) {
        { k_pack_rows<<<nb, 256, 0, s>>>(n, diag, nbr, w.rec); bnn_note_launch(); }
        rec = w.rec;
        if(coef) {
            // off-diagonal values ride along as 2 float4 per row
            if(!w.coefRow) BNN_CUDA_CHECK(dev_alloc(&w.coefRow, 2 * (size_t)w.cap * sizeof(float4)));
            { k_pack_coef<<<nb, 256, 0, s>>>(n, coef, w.coefRow); bnn_note_launch(); }
            coefRow = w.coefRow;
        }
    }
    if(mode == BNN_PCG_FP32) {
        rc = pcg_solve_t<float>(w, n, rhs, diag, invd, nbr, rec, coef, coefRow, -(1.0f * dt), tol, maxIter, w.x, w.r, w.z, w.s0, w.s1,
                                w.q, w.partMaxF, two, dst, hst, s, out);
        if(rc != BNN_OK) return rc;
        if(n > 0) BNN_CUDA_CHECK(cudaMemcpyAsync(pressure, w.x, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        if(x64out && n > 0) { k_f32_to_f64<<<nb, 256, 0, s>>>(n, w.x, x64out); bnn_note_launch(); }
        return BNN_OK;
    }
    if(mode == BNN_PCG_FP64) {
        if(n > 0) { k_inv_diag64<<<nb, 256, 0, s>>>(n, diag, w.inv64); bnn_note_launch(); }
        rc = pcg_solve_t<double>(w, n, rhs, diag, w.inv64, nbr, rec, coef, coefRow, -(double)(1.0f * dt), (double)tol, maxIter, w.x64,
                                 w.r64, w.z64, w.s064, w.s164, w.q64, w.partMaxD, two, dst, hst, s, out);
        if(rc != BNN_OK) return rc;
        if(n > 0) { k_d64_to_f32<<<nb, 256, 0, s>>>(n, w.x64, pressure); bnn_note_launch(); }
        if(x64out && n > 0)
            BNN_CUDA_CHECK(cudaMemcpyAsync(x64out, w.x64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        return BNN_OK;
    }
    // refined: FP64 outer residual and solution, FP32 inner solves
    if(n == 0) { out.success = 1; return BNN_OK; }
    { k_ir_init<<<nch, kLanes, 0, s>>>(n, rhs, w.x64, w.r64, w.partMaxD, dst); bnn_note_launch(); }
    BNN_CUDA_CHECK(cudaMemcpyAsync(hst, dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    const double bmax = hst->outer_bmax;
    unsigned total = 0, outer = 0;
    float kernelMs = 0.f;
    const unsigned maxOuter = 60;
    double res = bmax;
    bool ok = bmax < (double)FLT_MIN;
    while(!ok && outer < maxOuter) {
        if(res < (double)outerTol * bmax) { ok = true; break; }
        { k_ir_to_f32<<<nb, 256, 0, s>>>(n, w.r64, w.r32); bnn_note_launch(); }
        PcgOutcome inner;
        rc = pcg_solve_t<float>(w, n, w.r32, diag, invd, nbr, rec, coef, coefRow, -(1.0f * dt), innerTol, maxIter, w.d32, w.r, w.z, w.s0,
                                w.s1, w.q, w.partMaxF, two, dst, hst, s, inner);
        if(rc != BNN_OK) return rc;
        total += inner.iterations;
        kernelMs += inner.kernelMs;
        { k_ir_accumulate<<<nb, 256, 0, s>>>(n, w.x64, w.d32); bnn_note_launch(); }
        { k_ir_residual<<<nch, kLanes, 0, s>>>(n, rhs, w.x64, w.r64, diag, nbr, coef, (double)(-(1.0f * dt)), w.partMaxD, dst); bnn_note_launch(); }
        BNN_CUDA_CHECK(cudaMemcpyAsync(hst, dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        BNN_CUDA_CHECK(cudaStreamSynchronize(s));
        res = hst->outer_res;
        ++outer;
        if(total >= maxIter) break;
    }
    if(!ok && res < (double)outerTol * bmax) ok = true;
    out.iterations = total;
    out.outer = outer;
    out.kernelMs = kernelMs;
    out.residual = res;
    out.success = ok ? 1 : 0;
    { k_d64_to_f32<<<nb, 256, 0, s>>>(n, w.x64, pressure); bnn_note_launch(); }
    if(x64out) BNN_CUDA_CHECK(cudaMemcpyAsync(x64out, w.x64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return BNN_OK;
}

// ---------------------------------------------------------------------------------
// Batched refinement: pcg_solve's BNN_PCG_REFINED loop for many scenes at once.  Every
// stage is one launch over the scenes still refining (each scene's blocks found through a
// per-scene block prefix, as the batched step kernels do); the inner FP32 solves of all of
// them are one k_pcg_batch launch.  The host keeps each scene's outer loop state and
// takes exactly the decisions the lone loop takes, from the same device values.
// ---------------------------------------------------------------------------------
struct IrScene {
    int n;
    const float* b;            // right-hand side
    double *x64, *r64;
    float *r32, *d32;
    const float* diag;
    const int32_t* nbr;
    int4* rec;                 // packed rows
    double negoff;             // (double)(-(1 * dt))
    double* partMax;
    DevState* st;
    float* pressure;
};
struct IrReport {
    double res, bmax;
    unsigned iter, flags, done, pad;
};
// Uploaded with every launch's tables: the barrier word and the unfinished-scene counters
struct BatchHeader {
    GridSync gs;
    unsigned remaining;
    unsigned flags;
    unsigned active;
};

__global__ void kb_pack_rows(const IrScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const IrScene& c = S[q];
    const int n = c.n;
    const int r = b.x * blockDim.x + threadIdx.x;
    if(r >= n) return;
    int32_t nb[6];
#pragma unroll
    for(int k = 0; k < 6; ++k) nb[k] = c.nbr[(size_t)k * n + r];
    const unsigned dyM = nb[1] >= 0 ? (unsigned)(r - nb[1]) : 0u, dyP = nb[4] >= 0 ? (unsigned)(nb[4] - r) : 0u;
    const unsigned dzM = nb[0] >= 0 ? (unsigned)(r - nb[0]) : 0u, dzP = nb[5] >= 0 ? (unsigned)(nb[5] - r) : 0u;
    int4 v;
    v.x = (int)(dyM | (dyP << 16));
    v.y = (int)(dzM | (nb[2] >= 0 ? 0x80000000u : 0u));
    v.z = (int)(dzP | (nb[3] >= 0 ? 0x80000000u : 0u));
    v.w = __float_as_int(c.diag[r]);
    c.rec[r] = v;
}
__global__ void __launch_bounds__(kLanes) kb_ir_init(const IrScene* __restrict__ S, const unsigned* __restrict__ P,
                                                     int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const IrScene& c = S[q];
    ir_init_body(b, c.n, c.b, c.x64, c.r64, c.partMax, c.st);
}
__global__ void kb_ir_to_f32(const IrScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const IrScene& c = S[q];
    const size_t e = (size_t)b.x * blockDim.x + threadIdx.x;
    if(e < (size_t)c.n) c.r32[e] = (float)c.r64[e];
}
__global__ void kb_ir_accumulate(const IrScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const IrScene& c = S[q];
    const size_t e = (size_t)b.x * blockDim.x + threadIdx.x;
    if(e < (size_t)c.n) c.x64[e] = c.x64[e] + (double)c.d32[e];
}
__global__ void __launch_bounds__(kLanes) kb_ir_residual(const IrScene* __restrict__ S,
                                                         const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const IrScene& c = S[q];
    ir_residual_body(b, c.n, c.b, c.x64, c.r64, c.diag, c.nbr, nullptr, c.negoff, c.partMax, c.st);
}
__global__ void kb_ir_finish(const IrScene* __restrict__ S, const unsigned* __restrict__ P, int ns) {
    int q;
    const Blk b = seg_blk(P, ns, q);
    const IrScene& c = S[q];
    const size_t e = (size_t)b.x * blockDim.x + threadIdx.x;
    if(e < (size_t)c.n) c.pressure[e] = (float)c.x64[e];
}
// one thread per scene: what the host's outer loop reads, plus the barrier's flags
__global__ void kb_ir_report(const IrScene* __restrict__ S, int ns, const BatchHeader* hdr,
                             IrReport* __restrict__ out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if(q < ns) {
        const DevState* st = S[q].st;
        out[q] = IrReport{st->outer_res, st->outer_bmax, st->iter, st->flags, st->done, 0u};
    }
    if(q == 0) out[ns] = IrReport{0.0, 0.0, 0u, hdr->flags, 0u, 0u};
}

namespace {
// Layout of the context's device blob (the same offsets in the pinned host mirror):
// header, IrScene[cap], BatchPcgScene[cap], the prefixes of 256-row blocks and of 2048-row
// chunks (cap + 1 each), then IrReport[cap + 1] (read back, not uploaded).
struct BatchLayout {
    size_t hdr, irs, bps, p256, pch, rep, up, total;
    explicit BatchLayout(int cap) {
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        const size_t pre = (size_t)(cap + 1) * sizeof(unsigned);
        hdr = 0;
        irs = al(sizeof(BatchHeader));
        bps = irs + al((size_t)cap * sizeof(IrScene));
        p256 = bps + al((size_t)cap * sizeof(BatchPcgScene));
        pch = p256 + al(pre);
        up = pch + al(pre);
        rep = up;
        total = rep + al((size_t)(cap + 1) * sizeof(IrReport));
    }
};
} // namespace

static int batch_reserve(BatchPcgCtx& ctx, int count) {
    if(count <= ctx.cap && ctx.dev) return BNN_OK;
    pcg_batch_release(ctx);
    const int cap = count < 64 ? 64 : count + count / 4;
    const BatchLayout L(cap);
    BNN_CUDA_CHECK(cudaMalloc(&ctx.dev, L.total));
    BNN_CUDA_CHECK(cudaMallocHost(&ctx.host, L.total));
    std::memset(ctx.host, 0, L.total);
    for(auto& e : ctx.ev) BNN_CUDA_CHECK(cudaEventCreate(&e));
    ctx.cap = cap;
    ctx.upBytes = L.up;
    ctx.blobBytes = L.total;
    return BNN_OK;
}

void pcg_batch_release(BatchPcgCtx& ctx) {
    if(ctx.dev) cudaFree(ctx.dev);
    if(ctx.host) cudaFreeHost(ctx.host);
    for(auto& e : ctx.ev)
        if(e) cudaEventDestroy(e);
    ctx = BatchPcgCtx();
}

int pcg_solve_batch_refined(BatchPcgCtx& ctx, BatchSolveItem* items, int count, cudaStream_t s) {
    constexpr unsigned kMaxOuter = 60;  // pcg_solve's outer limit
    struct Outer {
        double bmax = 0, res = 0;
        unsigned outer = 0, total = 0;
        bool ok = false, stopped = false;
        float kernelMs = 0.f;
    };
    std::vector<int> live;
    for(int i = 0; i < count; ++i) {
        items[i].out = PcgOutcome();
        if(items[i].n == 0) { items[i].out.success = 1; continue; }
        const int rc = pcg_reserve(*items[i].w, items[i].n, true);
        if(rc != BNN_OK) return rc;
        live.push_back(i);
    }
    if(live.empty()) return BNN_OK;
    int rc = batch_reserve(ctx, (int)live.size());
    if(rc != BNN_OK) return rc;
    const BatchLayout L(ctx.cap);
    char* H = (char*)ctx.host;
    char* D = (char*)ctx.dev;
    BatchHeader* hh = (BatchHeader*)(H + L.hdr);
    IrScene* hirs = (IrScene*)(H + L.irs);
    BatchPcgScene* hbps = (BatchPcgScene*)(H + L.bps);
    unsigned* hp256 = (unsigned*)(H + L.p256);
    unsigned* hpch = (unsigned*)(H + L.pch);
    const IrReport* hrep = (const IrReport*)(H + L.rep);
    const IrScene* dirs = (const IrScene*)(D + L.irs);
    const unsigned* dp256 = (const unsigned*)(D + L.p256);
    const unsigned* dpch = (const unsigned*)(D + L.pch);
    BatchHeader* dh = (BatchHeader*)(D + L.hdr);
    IrReport* drep = (IrReport*)(D + L.rep);

    // tables for the scenes `set` (positions in items), uploaded in one copy; resume: the
    // inner solves carry on from a yield
    auto upload = [&](const std::vector<int>& set, bool resume = false) -> cudaError_t {
        hp256[0] = hpch[0] = 0;
        for(size_t k = 0; k < set.size(); ++k) {
            const BatchSolveItem& it = items[set[k]];
            PcgWork& w = *it.w;
            const int n = it.n;
            hirs[k] = IrScene{n, it.rhs, w.x64, w.r64, w.r32, w.d32, it.diag, it.nbr, w.rec,
                              (double)(-(1.0f * it.dt)), w.partMaxD, it.dst, it.pressure};
            BatchPcgScene& b = hbps[k];
            b.n = n; b.rhsF = w.r32; b.invd = it.invd; b.rec = w.rec; b.negoff = -(1.0f * it.dt);
            b.tolFactor = it.innerTol; b.maxIter = it.maxIter; b.x = w.d32; b.r = w.r; b.z = w.z; b.s0 = w.s0;
            b.s1 = w.s1; b.q = w.q; b.part0 = w.part; b.part1 = w.part + w.nchCap;
            b.part2 = w.part + 2 * (size_t)w.nchCap; b.partMax = w.partMaxF; b.dst = it.dst;
            b.resume = resume ? 1 : 0;
            hp256[k + 1] = hp256[k] + (unsigned)((n + 255) / 256);
            hpch[k + 1] = hpch[k] + (unsigned)((n + kChunk - 1) / kChunk);
        }
        *hh = BatchHeader{GridSync{0u}, (unsigned)set.size(), 0u, hpch[set.size()]};
        return cudaMemcpyAsync(D, H, L.up, cudaMemcpyHostToDevice, s);
    };
    auto report = [&](int ns) -> int {
        { kb_ir_report<<<(ns + 128) / 128, 128, 0, s>>>(dirs, ns, dh, drep); bnn_note_launch(); }
        BNN_CUDA_CHECK(cudaMemcpyAsync(H + L.rep, drep, (size_t)(ns + 1) * sizeof(IrReport), cudaMemcpyDeviceToHost, s));
        BNN_CUDA_CHECK(cudaStreamSynchronize(s));
        if(hrep[ns].flags & BNN_FLAG_TIMEOUT) { bnn_set_error("batched PCG grid barrier timed out"); return BNN_ERR_TIMEOUT; }
        return BNN_OK;
    };

    // outer loop start of every scene: x64 = 0, r64 = b, bmax
    std::vector<Outer> o(count);
    const int nl = (int)live.size();
    BNN_CUDA_CHECK(upload(live));
    { kb_pack_rows<<<hp256[nl], 256, 0, s>>>(dirs, dp256, nl); bnn_note_launch(); }
    { kb_ir_init<<<hpch[nl], kLanes, 0, s>>>(dirs, dpch, nl); bnn_note_launch(); }
    rc = report(nl);
    if(rc != BNN_OK) return rc;
    for(int k = 0; k < nl; ++k) {
        Outer& e = o[live[k]];
        e.bmax = hrep[k].bmax;
        e.res = hrep[k].res;
        e.ok = e.bmax < (double)FLT_MIN;
    }

    // cooperative grid of the inner solves
    int numSM = 0, perSMv = 0;
    {
        std::lock_guard<std::mutex> lk(g_coop.mu);
        if(!g_coop.numSM) {
            int dev = 0;
            BNN_CUDA_CHECK(cudaGetDevice(&dev));
            BNN_CUDA_CHECK(cudaDeviceGetAttribute(&g_coop.numSM, cudaDevAttrMultiProcessorCount, dev));
        }
        if(!g_coop.perSM[15]) {
            BNN_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_coop.perSM[15], k_pcg_batch, kLanes, 0));
            if(g_coop.perSM[15] < 1) { bnn_set_error("batched PCG kernel cannot be resident"); return BNN_ERR_CUDA; }
        }
        numSM = g_coop.numSM;
        perSMv = g_coop.perSM[15];
    }

    std::vector<int> set;
    for(;;) {
        // the lone loop's decisions, scene by scene
        set.clear();
        for(int i : live) {
            Outer& e = o[i];
            if(e.ok || e.stopped || e.outer >= kMaxOuter) continue;
            if(e.res < (double)items[i].outerTol * e.bmax) { e.ok = true; continue; }
            set.push_back(i);
        }
        if(set.empty()) break;
        const int ns = (int)set.size();
        BNN_CUDA_CHECK(upload(set));
        { kb_ir_to_f32<<<hp256[ns], 256, 0, s>>>(dirs, dp256, ns); bnn_note_launch(); }
        // the inner solves: launched over the whole grid, again for the scenes still
        // iterating whenever their chunks have fallen to half of a launch's
        float ms = 0.f;
        {
            std::vector<int> part = set;
            bool resume = false;
            for(;;) {
                const int np = (int)part.size();
                const unsigned total = hpch[np];
                const unsigned capB = (unsigned)(numSM * perSMv);
                // chunks striped over every resident block; a block's chunks (and so the
                // scenes it meets) must fit its slot table
                const unsigned grid = std::min(total, capB);
                const unsigned perBlock = (total + grid - 1) / grid;
                if(perBlock > (unsigned)kBatchSlots) {
                    bnn_set_error("batched PCG: too many chunks per block");
                    return BNN_ERR_CAPACITY;
                }
                BatchPcgArgs a;
                a.sc = (const BatchPcgScene*)(D + L.bps);
                a.cp = dpch;
                a.ns = np;
                a.total = total;
                a.perBlock = perBlock;
                a.gs = &dh->gs;
                a.remaining = &dh->remaining;
                a.active = &dh->active;
                a.yieldBelow = 0u;  // striped chunks stay balanced: no relaunch
                a.flags = &dh->flags;
                void* args[] = {(void*)&a};
                {
                    CoopShare share(grid * (kShareUnits / perSMv), numSM * kShareUnits);
                    BNN_CUDA_CHECK(cudaEventRecord(ctx.ev[0], s));
                    BNN_CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)k_pcg_batch, dim3(grid), dim3(kLanes), args, 0, s));
                    bnn_note_launch();
                    BNN_CUDA_CHECK(cudaEventRecord(ctx.ev[1], s));
                    rc = report(np);
                    if(rc != BNN_OK) return rc;
                }
                float lm = 0.f;
                cudaEventElapsedTime(&lm, ctx.ev[0], ctx.ev[1]);
                ms += lm;
                std::vector<int> left;
                for(int k = 0; k < np; ++k)
                    if(!hrep[k].done) left.push_back(part[k]);
                if(left.empty()) break;
                part.swap(left);
                resume = true;
                BNN_CUDA_CHECK(upload(part, resume));
            }
        }
        BNN_CUDA_CHECK(upload(set));
        { kb_ir_accumulate<<<hp256[ns], 256, 0, s>>>(dirs, dp256, ns); bnn_note_launch(); }
        { kb_ir_residual<<<hpch[ns], kLanes, 0, s>>>(dirs, dpch, ns); bnn_note_launch(); }
        rc = report(ns);
        if(rc != BNN_OK) return rc;
        for(int k = 0; k < ns; ++k) {
            Outer& e = o[set[k]];
            e.total += hrep[k].iter;
            e.kernelMs += ms;
            e.res = hrep[k].res;
            ++e.outer;
            if(e.total >= items[set[k]].maxIter) e.stopped = true;
        }
    }
    for(int i : live) {
        Outer& e = o[i];
        if(!e.ok && e.res < (double)items[i].outerTol * e.bmax) e.ok = true;
        PcgOutcome& out = items[i].out;
        out.iterations = e.total;
        out.outer = e.outer;
        out.kernelMs = e.kernelMs;
        out.residual = e.res;
        out.success = e.ok ? 1 : 0;
    }
    // pressure = (float) x64
    BNN_CUDA_CHECK(upload(live));
    { kb_ir_finish<<<hp256[nl], 256, 0, s>>>(dirs, dp256, nl); bnn_note_launch(); }
    BNN_CUDA_CHECK(cudaGetLastError());
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    return BNN_OK;
}

// ---- self-test of the bounded barrier wait -------------------------------------------
// One block arrives at a barrier sized for two blocks, so the wait can only end by giving
// up; out[0] = 1 when it gave up, out[1] = the block's polling time in ns.
__global__ void k_barrier_probe(GridSync* gs, unsigned* flags, BarrierLimit lim, unsigned long long* out) {
    unsigned sense = 0;
    const unsigned long long t0 = global_ns();
    const bool passed = grid_barrier(gs, 2u, sense, flags, lim);
    if(threadIdx.x == 0) {
        out[0] = passed ? 0ull : 1ull;
        out[1] = global_ns() - t0;
    }
}

int pcg_barrier_probe(float limitSeconds, int* barrierStatus, float* elapsedMs) {
    GridSync* gs = nullptr;
    unsigned* flags = nullptr;
    unsigned long long* out = nullptr;
    int rc = BNN_OK;
    auto chk = [&](cudaError_t e) { if(e != cudaSuccess && rc == BNN_OK) { bnn_set_error(cudaGetErrorString(e)); rc = e == cudaErrorMemoryAllocation ? BNN_ERR_OUT_OF_MEMORY : BNN_ERR_CUDA; } };
    chk(cudaMalloc(&gs, sizeof(GridSync)));
    chk(cudaMalloc(&flags, sizeof(unsigned)));
    chk(cudaMalloc(&out, 2 * sizeof(unsigned long long)));
    unsigned long long h[2] = {0, 0};
    unsigned hf = 0;
    if(rc == BNN_OK) {
        chk(cudaMemset(gs, 0, sizeof(GridSync)));
        chk(cudaMemset(flags, 0, sizeof(unsigned)));
    }
    if(rc == BNN_OK) {
        // 4096 polls, then limitSeconds of time; 2^26 polls at most whatever the clock says
        const BarrierLimit lim = {(unsigned long long)((double)limitSeconds * 1e9), 1u << 12, 1u << 26};
        k_barrier_probe<<<1, kLanes>>>(gs, flags, lim, out);
        bnn_note_launch();
        chk(cudaGetLastError());
        chk(cudaDeviceSynchronize());
        chk(cudaMemcpy(h, out, sizeof(h), cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(&hf, flags, sizeof(hf), cudaMemcpyDeviceToHost));
    }
    cudaFree(gs);
    cudaFree(flags);
    cudaFree(out);
    if(rc != BNN_OK) return rc;
    *barrierStatus = (h[0] == 1ull && (hf & BNN_FLAG_TIMEOUT)) ? BNN_ERR_TIMEOUT : BNN_OK;
    *elapsedMs = (float)((double)h[1] * 1e-6);
    return BNN_OK;
}

} // namespace bnn
