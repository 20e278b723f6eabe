// Internal declarations shared by the CUDA translation units of libbanana_b200.
//
// Arithmetic rule for every kernel here: the library is compiled with -fmad=false and
// IEEE division / square root, so each float operation rounds once, in the order it is
// written.  The expressions below follow the reference's own evaluation order (each
// device function cites the reference lines it computes), which is what lets the FLIP
// step agree bit for bit with a serial run of the reference's CPU code.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <cfloat>

#include "banana_b200.h"

namespace bnn {

// ----------------------------------------------------------------------------------
// Canonical reduction layout: a vector is cut into 2048-element chunks, one 256-thread
// block per chunk, thread t sums elements t, t+256, ... t+1792 of its chunk in FP64,
// then a halving tree (128, 64, ..., 1).  Chunk partials are reduced the same way by
// one block.  The result therefore depends only on n, never on the launch shape.
// ----------------------------------------------------------------------------------
constexpr int kLanes = 256;
constexpr int kPerLane = 8;
constexpr int kChunk = kLanes * kPerLane;

__device__ __forceinline__ double block_sum_256(double v, double* sm) {
    const int t = threadIdx.x;
    sm[t] = v;
    __syncthreads();
#pragma unroll
    for(int off = 128; off >= 32; off >>= 1) {
        if(t < off) sm[t] = sm[t] + sm[t + off];
        __syncthreads();
    }
    double r = 0.0;
    if(t < 32) {
        r = sm[t];
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) r = r + __shfl_down_sync(0xffffffffu, r, off);
    }
    __syncthreads();
    return r; // valid in thread 0
}

__device__ __forceinline__ float block_max_256(float v, float* sm) {
    const int t = threadIdx.x;
    sm[t] = v;
    __syncthreads();
    for(int off = 128; off >= 32; off >>= 1) {
        if(t < off) { float o = sm[t + off]; sm[t] = sm[t] > o ? sm[t] : o; }
        __syncthreads();
    }
    float r = 0.f;
    if(t < 32) {
        r = sm[t];
        for(int off = 16; off > 0; off >>= 1) {
            float o = __shfl_down_sync(0xffffffffu, r, off);
            r = r > o ? r : o;
        }
    }
    __syncthreads();
    return r;
}

// Last-block-done: every block publishes its partial, then the block that arrives last
// reduces all partials in the fixed order.  The counter is reset by that block.
__device__ __forceinline__ bool last_block(unsigned* counter) {
    __shared__ bool amLast;
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0) {
        unsigned prev = atomicAdd(counter, 1u);
        amLast = (prev == gridDim.x - 1);
    }
    __syncthreads();
    return amLast;
}

// Final pass over chunk partials in the canonical order (called by one whole block);
// the result is returned to every thread of the block.
__device__ __forceinline__ double reduce_partials(const double* part, int nch, double* sm) {
    double acc = 0.0;
    for(int c = threadIdx.x; c < nch; c += kLanes) acc = acc + __ldcg(part + c);
    const double r = block_sum_256(acc, sm);
    if(threadIdx.x == 0) sm[0] = r;
    __syncthreads();
    const double b = sm[0];
    __syncthreads();
    return b;
}
__device__ __forceinline__ float reduce_partials_max(const float* part, int nch, float* sm) {
    float acc = 0.f;
    for(int c = threadIdx.x; c < nch; c += kLanes) { float o = __ldcg(part + c); acc = acc > o ? acc : o; }
    return block_max_256(acc, sm);
}

// Block coordinates a kernel body works in: its own launch's (blockIdx.x, gridDim.x), or,
// in a batched launch over many scenes (batch_step.cu), the block's place within its
// scene's share of the launch.
struct Blk {
    unsigned x, n;
};
__device__ __forceinline__ Blk own_blk() { return Blk{blockIdx.x, gridDim.x}; }

// The segment (scene) a block of a batched launch belongs to: prefix[s] <= b < prefix[s+1],
// prefix[0] = 0, prefix[nseg] = the launch's blocks (segments with no blocks are skipped).
__device__ __forceinline__ int seg_of(const unsigned* __restrict__ prefix, int nseg, unsigned b) {
    int lo = 0, hi = nseg;
    while(hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if(__ldg(prefix + mid) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}
// The block's segment and its place within the segment's blocks
__device__ __forceinline__ Blk seg_blk(const unsigned* __restrict__ prefix, int nseg, int& s) {
    s = seg_of(prefix, nseg, blockIdx.x);
    const unsigned b0 = __ldg(prefix + s);
    return Blk{blockIdx.x - b0, __ldg(prefix + s + 1) - b0};
}
// Batched element-wise stages give a block kBatchVirt consecutive blocks of the lone
// launch's layout (virtual blocks), so the cost of finding the scene is paid once per
// kBatchVirt blocks of work.  f(Blk) runs the lone body for virtual blocks
// b.x * kBatchVirt + j below `count` (the scene's lone block count), in order.
constexpr unsigned kBatchVirt = 8;
template<class F> __device__ __forceinline__ void virtual_blocks(Blk b, unsigned count, F f) {
#pragma unroll 1
    for(unsigned j = 0; j < kBatchVirt; ++j) {
        const unsigned v = b.x * kBatchVirt + j;
        if(v >= count) break;
        f(Blk{v, count});
    }
}

// ----------------------------------------------------------------------------------
// Scalar helpers, same semantics as the reference's MathHelpers
// ----------------------------------------------------------------------------------
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; } // std::min
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; } // std::max

// MathHelpers::get_barycentric(x, i, f, 0, i_high) (MathHelpers.h:516-530)
__device__ __forceinline__ void bary(float x, int& i, float& f, int i_high) {
    float s = floorf(x);
    i = (int)s;
    if(i < 0) { i = 0; f = 0.f; }
    else if(i > i_high - 2) { i = i_high - 2; f = 1.f; }
    else { f = x - s; }
}
// MathHelpers::lerp (MathHelpers.h:549-551)
__device__ __forceinline__ float lerpf(float v0, float v1, float f) { return (1.0f - f) * v0 + f * v1; }
// MathHelpers::fraction_inside(left, right) (MathHelpers.h:823-838)
__device__ __forceinline__ float fraction_inside(float l, float r) {
    if(l < 0.f && r < 0.f) return 1.0f;
    if(l < 0.f && r >= 0.f) return l / (l - r);
    if(l >= 0.f && r < 0.f) return r / (r - l);
    return 0.f;
}
__device__ __forceinline__ float length2f(float x, float y, float z) { return (x * x + y * y) + z * z; }

// A boundary object (BoundaryObject over GeometryObjects::BoxObject / SphereObject,
// Simulation/SimulationObjects/BoundaryObject.h:41-60, GeometryObjects.cpp:221-268,379-384):
// the signed distance with bNegativeInside = false, i.e. positive inside the object,
// which bounds the fluid.
struct BObj {
    int geometry;      // 0 box, 1 sphere (unit sphere in object space)
    int transformed;   // 0: invTransform is the identity and is skipped
    float bmin[3], bmax[3];
    float M[12];       // world -> object: rows of a 3x4 affine map
    float scale;       // uniform scale (multiplies the object-space distance)
};
constexpr int kMaxBoundaryObjects = 16;

// Grid description passed by value to kernels
struct GridDesc {
    int G[3];          // cells per axis (after padding)
    float dx;          // cell size
    float bmin[3];     // padded domain min
    float boxMin[3];   // domain box (constraint) min
    float boxMax[3];   // domain box max
    float sdfRadius;   // PIC_Parameters::sdfRadius
    // Boundary objects beyond the plain domain box (nObj = 0: the domain box alone, above).
    // obj[0, nStatic) are the static objects, the domain box first, united into one CSG
    // object; every later object is a dynamic one of its own.
    const BObj* obj = nullptr;
    int nObj = 0;
    int nStatic = 0;
};

// GeometryObject::invTransform then BoxObject / SphereObject::signedDistance(p, false)
__device__ __forceinline__ float bobj_sdf(const BObj& o, float x, float y, float z) {
    float q[3] = {x, y, z};
    if(o.transformed) {
#pragma unroll
        for(int r = 0; r < 3; ++r) q[r] = ((o.M[4 * r] * x + o.M[4 * r + 1] * y) + o.M[4 * r + 2] * z) + o.M[4 * r + 3];
    }
    if(o.geometry == 0) {
        bool inside = true;
#pragma unroll
        for(int d = 0; d < 3; ++d)
            if(q[d] < o.bmin[d] || q[d] > o.bmax[d]) inside = false;
        float mind = 3.402823466e+38f;
        if(inside) {
#pragma unroll
            for(int d = 0; d < 3; ++d) mind = smin(mind, smin(q[d] - o.bmin[d], o.bmax[d] - q[d]));
            mind = -mind;
        } else {
            float c[3];
#pragma unroll
            for(int d = 0; d < 3; ++d) c[d] = smax(smin(q[d], o.bmax[d]), o.bmin[d]);
            mind = sqrtf(length2f(q[0] - c[0], q[1] - c[1], q[2] - c[2]));
        }
        mind = -mind;
        return o.scale * mind;
    }
    const float d = o.scale * (sqrtf(length2f(q[0], q[1], q[2])) - 1.0f);
    return -d;
}

// Signed distance of boundary group grp: group 0 is the CSG union of the static objects
// (CSGObject::signedDistance, GeometryObjects.cpp:861-896: min over the members in
// order), group g > 0 the g-th dynamic object
__device__ __forceinline__ float group_sdf(const GridDesc& g, int grp, float x, float y, float z) {
    const int b = grp == 0 ? 0 : g.nStatic + grp - 1;
    const int e = grp == 0 ? g.nStatic : b + 1;
    float sd = bobj_sdf(g.obj[b], x, y, z);
    for(int i = b + 1; i < e; ++i) sd = smin(sd, bobj_sdf(g.obj[i], x, y, z));
    return sd;
}

__host__ __device__ __forceinline__ int face_sx(const GridDesc& g, int d) { return g.G[0] + (d == 0); }
__host__ __device__ __forceinline__ int face_sy(const GridDesc& g, int d) { return g.G[1] + (d == 1); }
__host__ __device__ __forceinline__ int face_sz(const GridDesc& g, int d) { return g.G[2] + (d == 2); }

// Device-side state of one solver: PCG scalars, reduction counters and check flags
struct DevState {
    // PCG
    double rho, tmp, dotv;
    double alpha64, beta64;
    float alpha, beta, resid, tol;
    double resid64, tol64;
    unsigned iter, done, success, max_iter;
    unsigned counter0, counter1, counter2, counter3;
    // step
    unsigned maxvel_bits;   // max |u| over faces as float bits (non-negative)
    unsigned flags;         // BNN device flags
    unsigned n_active;
    unsigned zero_phi;
    unsigned out_of_range;
    unsigned pad0;
    double outer_res, outer_bmax;
    int bbox[6];            // min x,y,z and max x,y,z of the particles' (clamped) cells
    unsigned nlarge;        // cells with more than 16 particles, listed for k_sort_large
    // the next sub-step, when its particle move ran at the end of this one (k_g2p_move)
    float next_dt;          // its size (PIC_Solver::advanceFrame's substep)
    unsigned next_flags;    // flags its move raised (BNN_FLAG_OUT_OF_GRID)
};

// What the fused grid-to-particle + move pass needs to size the next sub-step
// (PIC_Solver::timestepCFL + advanceFrame's clipping, PIC_Solver.cpp:284-290,342-349) on
// the device: the frame time after this sub-step and the parameters.
struct NextStep {
    float frameTime;        // frameLocalTime after this sub-step (before the new-frame wrap)
    float frameDuration;
    float cfl, minDt, maxDt;
    int advSteps;
};

#define BNN_FLAG_OUT_OF_GRID   1u
#define BNN_FLAG_RING_FLUID    2u
#define BNN_FLAG_PCG_MAXITER   4u
#define BNN_FLAG_SCRATCH_LIMIT 8u
#define BNN_FLAG_TIMEOUT       16u

// ----------------------------------------------------------------------------------
// One scene of a batched sub-step (batch_step.cu): what its stage kernels read.  The
// batched kernels run the same bodies as a lone scene's kernels, each block on the scene
// and block coordinates its place in the launch gives it (seg_blk).
// ----------------------------------------------------------------------------------
struct BScene {
    GridDesc g;
    int n;                  // particles
    int nrows;              // pressure rows (known after the system's numbering)
    int advSteps;
    int moved;              // the move already ran at the end of the last sub-step
    size_t cap;             // particle plane stride
    size_t C;               // cells
    float sub, substep, gdt;
    float ratio;            // PIC_FLIP_ratio
    NextStep ns;            // the next sub-step (fused move)
    float *p6cur, *p6nxt, *movedPos;
    uint32_t *idcur, *idnxt;
    float4* rec;
    uint32_t *cellOf, *slot, *order, *key, *count, *cellStart;
    int* bboxPart;
    float* U[3];
    float* B[3];
    float* O[3];
    uint8_t* VA[3];
    uint8_t* VB[3];
    float* phi;
    uint32_t *flag, *aidx, *rowCell;
    float *rhs, *diag, *invd, *pressure;
    int32_t* nbr;
    DevState* dst;
};
// Stages of the batched sub-step (flip_kernels.cu), one launch each over all scenes
enum class BatchStage {
    StepReset, BboxReset, Advect, BboxFinal, ScatterIndex, SortBuckets, SortLarge, Gather, FillBackup, FillUpdate,
    Extrapolate, ActiveFlags, ActiveRows, BuildRows, UpdateU, UpdateV, UpdateW, G2PMove
};
void launch_batch_stage(BatchStage stage, const BScene* S, const unsigned* P, int ns, unsigned blocks, cudaStream_t s,
                        int pass = 0, int layer = 0);
void launch_batch_gather_rows(const BScene* S, int ns, unsigned* out, cudaStream_t s);
void launch_batch_gather_state(const BScene* S, int ns, DevState* out, cudaStream_t s);
// The FLIP P2G + fluid SDF pass of all scenes (gather_kernels.cu): per-scene argument
// records (p2g_tile_args, p2g_tile_args_bytes() each) and the tile prefix P
// in each tile shape (launch_p2g_sdf_batch picks one: P[shape] and tiles[shape] are the
// tile prefix and total of every shape, cells the batch's total cells)
constexpr int kTileShapes = 6;
unsigned p2g_sdf_tiles(const GridDesc& g, int shape);
size_t p2g_tile_args_bytes();
void p2g_tile_args(void* out, const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                   size_t stride, float* const U[3], uint8_t* const valid[3], float* phi);
void launch_p2g_sdf_batch(const void* args, const unsigned* const* P, const unsigned* tiles, int ns, uint64_t cells,
                          cudaStream_t s);
// The shape launch_p2g_sdf_batch will use for such a batch, or -1 while it is untuned (its
// next call then times every shape and synchronises the stream); also opts every batched
// shape into its shared memory, so a launch can be captured into a graph
int p2g_batch_shape(int ns, uint64_t cells);
// The tile-shape tuner (gather_kernels.cu): force a shape for every launch (-1: tune), the
// dimensions of a shape, and the table of tuned choices as JSON lines
int tile_shape_set(int shape);
void tile_shape_dims(int shape, int* tz, int* yc);

// ----------------------------------------------------------------------------------
// Host-side launchers (defined in the .cu files)
// ----------------------------------------------------------------------------------
// scan.cu
size_t scan_workspace_bytes(size_t n);
// exclusive scan of n uint32 into out[0..n], out[n] = total; ws from scan_workspace_bytes
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, void* ws, cudaStream_t s);
// Many independent exclusive scans in three launches: segment q scans in[0..n) into
// out[0..n] with workspace ws (scan_workspace_bytes(n)); in and out 16-byte aligned.
// tiles[q] is the prefix of the segments' kScanSegTile-element tile counts (at least 1
// each; tiles[nseg] = totalTiles), in device memory.
constexpr unsigned kScanSegTile = 16384;
struct ScanSeg {
    const uint32_t* in;
    uint32_t* out;
    uint32_t* ws;
    size_t n;
};
cudaError_t batched_exclusive_scan_u32(const ScanSeg* segs, const unsigned* tiles, int nseg, unsigned totalTiles,
                                       cudaStream_t s);

// pcg.cu
struct GridSync {
    unsigned count;  // arrivals at the current barrier (top bit: barriers passed, mod 2)
};
struct PcgWork {
    int cap = 0;
    int nchCap = 0;
    GridSync* gs = nullptr;
    float *x = nullptr, *r = nullptr, *z = nullptr, *s0 = nullptr, *s1 = nullptr, *q = nullptr, *d32 = nullptr,
          *r32 = nullptr;
    double *x64 = nullptr, *r64 = nullptr, *z64 = nullptr, *s064 = nullptr, *s164 = nullptr, *q64 = nullptr,
           *inv64 = nullptr;
    double* part = nullptr;
    float* partMaxF = nullptr;
    double* partMaxD = nullptr;
    int4* rec = nullptr;  // packed grid rows
    float4* coefRow = nullptr;  // packed rows' off-diagonal values (2 per row)
    // single-reduction solve: row records {r, w, s, 1/diag} (double-buffered; FP32 as
    // float4, FP64 as 4 doubles) and the partials of both sums and the max (double-buffered)
    float4* st32[2] = {nullptr, nullptr};
    double* st64[2] = {nullptr, nullptr};
    double* cgPart = nullptr;  // [2][2][nchCap]
    double* cgMax = nullptr;   // [2][nchCap]
    cudaEvent_t ev[2] = {nullptr, nullptr};  // around the persistent launch
};
struct PcgOutcome {
    unsigned iterations = 0, outer = 0, success = 0;
    double residual = 0;
    float kernelMs = 0.f;  // device time of the persistent launches (all inner solves)
};
// gridRows: the x neighbours of every row are rows r-1 / r+1 (or none) and the y
// neighbours lie within 65535 rows (rows of a grid in cell order, at most 65535 cells
// along x); the solve then reads the packed 16-byte row records.
// coef (optional): six planes of off-diagonal values in the order of nbr (face weights
// != 1); without it every off-diagonal is -dt.
int pcg_solve(PcgWork& w, int n, const float* rhs, const float* diag, const float* invd, const int32_t* nbr,
              const float* coef, bool gridRows, float dt, int mode, float tol, unsigned maxIter, float innerTol,
              float outerTol, float* pressure, double* x64out, DevState* dst, DevState* hst, cudaStream_t s,
              PcgOutcome& out);
int pcg_reserve(PcgWork& w, int n, bool fp64);
// One scene's system in a batched refined solve (BNN_PCG_REFINED, two-reduction steps,
// rows of a grid, face weights 1): what pcg_solve would be called with, and its outcome.
struct BatchSolveItem {
    PcgWork* w;
    int n;
    const float *rhs, *diag, *invd;
    const int32_t* nbr;
    float dt, innerTol, outerTol;
    unsigned maxIter;
    float* pressure;
    DevState* dst;
    PcgOutcome out;
};
// Device tables of the batched solve, kept between calls (grown on demand)
struct BatchPcgCtx {
    int cap = 0;
    size_t upBytes = 0, blobBytes = 0;
    void* dev = nullptr;       // device tables, reports, barrier
    void* host = nullptr;      // pinned mirror of the uploaded part, then the reports
    cudaEvent_t ev[2] = {nullptr, nullptr};
};
// The refined solves of many scenes, each stage one launch over the scenes still
// refining: every scene gets exactly what pcg_solve gives it alone.  Returns BNN status;
// items[i].out holds each scene's outcome, its pressure is written.
int pcg_solve_batch_refined(BatchPcgCtx& ctx, BatchSolveItem* items, int count, cudaStream_t s);
void pcg_batch_release(BatchPcgCtx& ctx);
// one block waits at a barrier sized for two until the bounded wait gives up
int pcg_barrier_probe(float limitSeconds, int* barrierStatus, float* elapsedMs);
// Cell grid of the anisotropic-kernel pass (aniso.cu)
struct AnisoGrid {
    int G[3];
    float dx;
    float bmin[3];
};
bnn_aniso_params aniso_defaults(float particleRadius);
int aniso_check_params(const bnn_aniso_params& p);
void launch_aniso(int n, const float4* pos, const uint32_t* ids, const uint32_t* cellStart, const AnisoGrid& g,
                  const bnn_aniso_params& prm, float* outC, float* outM, unsigned* counters, cudaStream_t s);

void pcg_release(PcgWork& w);

} // namespace bnn

extern "C" void bnn_set_error(const char* msg);

// Device memory of solver handles (grids, particles, rows, PCG vectors) comes from the
// device's stream-ordered memory pool: allocating and freeing a scene's arrays then costs
// neither a driver allocation each nor, on free, a synchronisation of the whole device
// (what cudaFree does) -- scenes come and go between the steps of a serving batch.  An
// allocation is usable on every stream when dev_alloc returns; dev_free requires that no
// work on the memory is pending (every API call that frees ends its streams' work first).
cudaError_t dev_alloc_bytes(void** p, size_t bytes);
// Sets up this device's stream-ordered memory pool (keeps freed memory for reuse) once
cudaError_t mem_pool_setup();
void dev_free_ptr(void* p);
template<class T> inline cudaError_t dev_alloc(T** p, size_t bytes) { return dev_alloc_bytes((void**)p, bytes); }
inline cudaError_t dev_free(const void* p) {
    dev_free_ptr(const_cast<void*>(p));
    return cudaSuccess;
}

// Every kernel launch of the library is followed by bnn_note_launch(): the running total
// is what bnn_launch_count() reports.  Launches captured into a CUDA graph are taken back
// (bnn_note_launches(-k)) and counted again at every replay (bnn_note_launches(k)).
void bnn_note_launch();
void bnn_note_launches(long long k);

#define BNN_CUDA_CHECK(expr)                                                                 \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if(_e != cudaSuccess) {                                                              \
            bnn_set_error(cudaGetErrorString(_e));                                           \
            return _e == cudaErrorMemoryAllocation ? BNN_ERR_OUT_OF_MEMORY : BNN_ERR_CUDA;   \
        }                                                                                    \
    } while(0)
