// C ABI of libbanana_b200: solver handle, memory, and the host-side order of one
// FLIP / APIC / AFLIP sub-step (PIC_Solver::advanceFrame, PIC_Solver.cpp:267-311, and
// FLIP_Solver::advanceVelocity, FLIP_Solver.cpp:42-53).
#include "bnn_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include <atomic>

static thread_local std::string g_lastError;
static std::atomic<unsigned long long> g_launches{0};
void bnn_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void bnn_note_launches(long long k) { g_launches.fetch_add((unsigned long long)k, std::memory_order_relaxed); }
extern "C" uint64_t bnn_launch_count(void) { return g_launches.load(); }
extern "C" void bnn_set_error(const char* msg) { g_lastError = msg ? msg : ""; }
extern "C" const char* bnn_last_error(void) { return g_lastError.c_str(); }
extern "C" const char* bnn_version(void) { return "banana_b200 0.1 (sm_100a)"; }

// The pool keeps up to 16 GB of freed memory for reuse instead of handing it back to the
// driver at every synchronisation; allocations and frees are ordered on the calling
// thread's default stream, which the handles never queue work on.
static std::atomic<uint64_t> g_poolSetUp{0};  // bit per device ordinal
cudaError_t mem_pool_setup() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if(e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if(!(g_poolSetUp.load(std::memory_order_acquire) & bit)) {
        cudaMemPool_t pool;
        if(cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = 16ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        g_poolSetUp.fetch_or(bit, std::memory_order_acq_rel);
    }
    return cudaSuccess;
}
cudaError_t dev_alloc_bytes(void** p, size_t bytes) {
    cudaError_t e = mem_pool_setup();
    if(e != cudaSuccess) return e;
    e = cudaMallocAsync(p, bytes ? bytes : 1, cudaStreamPerThread);
    if(e != cudaSuccess) return e;
    return cudaStreamSynchronize(cudaStreamPerThread);
}
void dev_free_ptr(void* p) {
    if(p) cudaFreeAsync(p, cudaStreamPerThread);
}

// Pinned host copies of the per-handle device record come from page-sized pinned blocks
// (cudaHostAlloc is a slow call; a handle needs one small record)
namespace {
struct PinnedStates {
    std::mutex mu;
    std::vector<bnn::DevState*> freeList;
};
PinnedStates& pinned_states() {
    static PinnedStates p;
    return p;
}
} // namespace
static cudaError_t pinned_state_alloc(bnn::DevState** out) {
    PinnedStates& P = pinned_states();
    std::lock_guard<std::mutex> lk(P.mu);
    if(P.freeList.empty()) {
        constexpr int kPer = 64;
        bnn::DevState* blk = nullptr;
        const cudaError_t e = cudaHostAlloc(&blk, kPer * sizeof(bnn::DevState), cudaHostAllocDefault);
        if(e != cudaSuccess) return e;
        for(int i = kPer - 1; i >= 0; --i) P.freeList.push_back(blk + i);
    }
    *out = P.freeList.back();
    P.freeList.pop_back();
    return cudaSuccess;
}
static void pinned_state_free(bnn::DevState* p) {
    if(!p) return;
    PinnedStates& P = pinned_states();
    std::lock_guard<std::mutex> lk(P.mu);
    P.freeList.push_back(p);
}

namespace bnn {
// flip_kernels.cu
void launch_advect(int n, float* p6, size_t stride, const float* const* U, const GridDesc& g, float sub, int steps,
                   uint32_t* cellOf, uint32_t* slot, uint32_t* count, DevState* st, int* bboxPart, cudaStream_t s);
void launch_cell_histogram(int n, const float* p6, size_t stride, const GridDesc& g, uint32_t* cellOf, uint32_t* slot,
                           uint32_t* count, DevState* st, cudaStream_t s);
void launch_sort_finish(int n, size_t ncells, uint32_t* cellOf, uint32_t* slot, const uint32_t* cellStart,
                        uint32_t* order, uint32_t* key, uint32_t* count, const float* src6, const float* srcPos,
                        float* dst6, const uint32_t* idSrc, uint32_t* idDst, const float* cSrc, float* cDst,
                        float4* rec, const GridDesc& g, size_t stride, DevState* st, cudaStream_t s,
                        cudaEvent_t gatherAfter = nullptr);
// gather_kernels.cu
void launch_p2g_sdf(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                    size_t stride, float* const* out, uint8_t* const* valid, float* phi, cudaStream_t s);
void launch_p2g_sdf_affine(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                           const float* C9, size_t stride, float* const* out, uint8_t* const* valid, float* phi,
                           cudaStream_t s);
void launch_fluid_sdf_tile(const GridDesc& g, const DevState* st, const uint32_t* cellStart, const float4* rec,
                           size_t stride, float* phi, cudaStream_t s);
void launch_advect_grid(const GridDesc& g, float** U, float** B, float dt, cudaStream_t s);
void launch_maxabs(const float* a, size_t n, unsigned* maxBits, cudaStream_t s);
void launch_correct_positions(int n, const GridDesc& g, const float* p6, size_t stride, const uint32_t* ids,
                              const uint32_t* cellStart, float radius2, float threshold2, float jitterScale,
                              float kSpring, int advSteps, unsigned long long step, float* out3, cudaStream_t s);
void launch_rebin(int n, const float* p6, size_t stride, const GridDesc& g, uint32_t* cellOf, uint32_t* slot,
                  uint32_t* count, DevState* st, cudaStream_t s);
void launch_extrapolate(const GridDesc& g, float* const* A, uint8_t* const* VA, float* const* B, uint8_t* const* VB,
                        int lastMode, float* const* oldOut, float gravityDt, DevState* st, cudaStream_t s);
void launch_active_flags(const GridDesc& g, const float* phi, uint32_t* flag, DevState* st, cudaStream_t s);
void launch_active_rows(size_t nc, const uint32_t* flag, const uint32_t* idx, uint32_t* rowCell, cudaStream_t s);
void launch_build_rows(const GridDesc& g, int nrows, const uint32_t* rowCell, const float* phi, const uint32_t* aidx,
                       const float* const* U, const float* const* W, float dt, float* rhs, float* diag, float* invdiag,
                       int32_t* nbr, float* coef, DevState* st, cudaStream_t s);
void launch_update_velocity(const GridDesc& g, const DevState* st, const float* phi, const uint32_t* aidx,
                            const float* pressure, float dt, float* const* velIn, float* const* velOut,
                            uint8_t* const* validOut, const float* const* W, cudaStream_t s);
void launch_g2p(int n, const GridDesc& g, float* p6, size_t stride, const float* const* U, const float* const* O,
                float ratio, int kind, float* C9, cudaStream_t s);
void launch_aos_to_soa(int n, const float* pos, const float* vel, float* soa6, uint32_t* ids, size_t stride,
                       cudaStream_t s);
void launch_soa_to_aos(int n, const float* soa6, const uint32_t* ids, float* pos, float* vel, size_t stride,
                       cudaStream_t s);
void launch_aos3_to_soa(int n, const float* aos, float* soa3, uint32_t* ids, size_t stride, cudaStream_t s);
void launch_boundary_grid(const GridDesc& g, float* nodeSdf, float* const* W, cudaStream_t s);
void launch_solid_extend(const GridDesc& g, const float* nodeSdf, float* phi, cudaStream_t s);
void launch_constrain_velocity(const GridDesc& g, const DevState* st, float* const* U, uint8_t* const* V,
                               float* const* W, const float* nodeSdf, float* const* T, cudaStream_t s);
void launch_soa3_to_aos(int n, const float* soa3, const uint32_t* ids, float* aos, size_t stride, cudaStream_t s);
void launch_scatter_planes(int n, int planes, const float* src, const uint32_t* ids, float* dst, size_t stride,
                           cudaStream_t s);
void launch_cells_from_rows(size_t nc, const float* phi, const uint32_t* aidx, const float* pr, float* out, int active,
                            cudaStream_t s);
void launch_add_scalar(float* a, size_t n, float v, cudaStream_t s);
void launch_step_reset(DevState* st, cudaStream_t s);
void launch_step_reset_moved(DevState* st, cudaStream_t s);
void launch_g2p_move(int n, const GridDesc& g, float* p6, size_t stride, const float* const* U, const float* const* O,
                     float ratio, int kind, float* C9, const NextStep& ns, float* moved, uint32_t* cellOf,
                     uint32_t* slot, uint32_t* count, DevState* st, int* bboxPart, cudaStream_t s);

// pcg.cu
} // namespace bnn

using namespace bnn;

#include "flip_handle.cuh"

static void free_particles(bnn_flip* h) {
    for(int b = 0; b < 2; ++b) {
        dev_free(h->p6[b]); dev_free(h->ids[b]); dev_free(h->C9[b]);
        h->p6[b] = nullptr; h->ids[b] = nullptr; h->C9[b] = nullptr;
    }
    dev_free(h->rec); dev_free(h->bboxPart); dev_free(h->cellOf); dev_free(h->slot); dev_free(h->order); dev_free(h->key); dev_free(h->aosStage);
    dev_free(h->aniso); dev_free(h->moved);
    h->rec = nullptr; h->bboxPart = nullptr; h->cellOf = h->slot = h->order = h->key = nullptr; h->aosStage = nullptr;
    h->aniso = nullptr; h->moved = nullptr;
    h->premoved = false;
    h->cap = 0;
}

static int reserve_particles(bnn_flip* h, uint32_t n) {
    if(n <= h->cap) return BNN_OK;
    free_particles(h);
    // a multiple of 64, so every plane of every particle array starts 256-byte aligned
    const uint64_t cap64 = ((uint64_t)n + 63u) & ~(uint64_t)63u;
    if(cap64 > 0xffffffffull) { bnn_set_error("too many particles"); return BNN_ERR_INVALID_ARGUMENT; }
    uint32_t cap = (uint32_t)cap64;
    size_t st = cap;
    for(int b = 0; b < 2; ++b) {
        BNN_CUDA_CHECK(dev_alloc(&h->p6[b], 6 * st * sizeof(float)));
        BNN_CUDA_CHECK(dev_alloc(&h->ids[b], st * sizeof(uint32_t)));
        if(h->P.solver_kind == BNN_SOLVER_APIC || h->P.solver_kind == BNN_SOLVER_AFLIP)
            BNN_CUDA_CHECK(dev_alloc(&h->C9[b], 9 * st * sizeof(float)));
    }
    // per-particle records of the P2G + SDF pass: 3 stencil planes and the positions
    BNN_CUDA_CHECK(dev_alloc(&h->rec, 4 * st * sizeof(float4)));
    BNN_CUDA_CHECK(dev_alloc(&h->bboxPart, 6 * ((st + 255) / 256) * sizeof(int)));
    BNN_CUDA_CHECK(dev_alloc(&h->cellOf, st * sizeof(uint32_t)));
    BNN_CUDA_CHECK(dev_alloc(&h->slot, st * sizeof(uint32_t)));
    BNN_CUDA_CHECK(dev_alloc(&h->order, st * sizeof(uint32_t)));
    BNN_CUDA_CHECK(dev_alloc(&h->key, st * sizeof(uint32_t)));
    BNN_CUDA_CHECK(dev_alloc(&h->aosStage, 6 * st * sizeof(float)));
    // positions moved for the next sub-step by the fused transfer + move (not PIC, which has no transfer)
    if(h->P.solver_kind != BNN_SOLVER_PIC) BNN_CUDA_CHECK(dev_alloc(&h->moved, 3 * st * sizeof(float)));
    h->cap = cap;
    return BNN_OK;
}

static void destroy_all(bnn_flip* h) {
    if(!h) return;
    free_particles(h);
    for(int d = 0; d < 3; ++d) {
        dev_free(h->U[d]); dev_free(h->B[d]); dev_free(h->O[d]); dev_free(h->VA[d]); dev_free(h->VB[d]);
    }
    dev_free(h->count); dev_free(h->cellStart); dev_free(h->scanWs); dev_free(h->phi); dev_free(h->flag);
    dev_free(h->aidx); dev_free(h->cellTmp);
    dev_free(h->rowCell); dev_free(h->rhs); dev_free(h->diag); dev_free(h->invd); dev_free(h->pressure); dev_free(h->nbr);
    pcg_release(h->pcg);
    dev_free(h->objDev); dev_free(h->nodeSdf); dev_free(h->coef);
    for(int d = 0; d < 3; ++d) dev_free(h->W[d]);
    dev_free(h->dst);
    pinned_state_free(h->hst);
    for(auto& e : h->ev) if(e) cudaEventDestroy(e);
    for(auto& e : h->io) if(e) cudaEventDestroy(e);
    if(h->s2) cudaStreamDestroy(h->s2);
    if(h->s) cudaStreamDestroy(h->s);
    delete h;
}

extern "C" int bnn_flip_create(const bnn_params* params, bnn_flip** out) {
    if(!params || !out) return BNN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const bnn_params& P = *params;
    if(!(P.cell_size > 0.f) || P.advection_steps == 0) return BNN_ERR_INVALID_ARGUMENT;
    if(P.solver_kind < 0 || P.solver_kind > 3) return BNN_ERR_NOT_SUPPORTED;
    if((P.pcg_mode & ~(BNN_PCG_MODE_MASK | BNN_PCG_SINGLE_REDUCTION)) != 0 || (P.pcg_mode & BNN_PCG_MODE_MASK) > 2 ||
       P.preconditioner != BNN_PRECOND_JACOBI)
        return BNN_ERR_NOT_SUPPORTED;
    for(int d = 0; d < 3; ++d) if(!(P.box_max[d] > P.box_min[d])) return BNN_ERR_INVALID_ARGUMENT;
    auto* h = new bnn_flip();
    h->P = P;
    // SimulationParameters::makeReady (ParticleSolverData.cpp:229-272), Grid::setCellSize
    // (Grid.cpp:38-55), PIC_Parameters::makeReady (PIC_Data.cpp:41-44)
    const float dx = P.cell_size;
    const float pad = dx * (float)P.n_expand_cells;
    h->g.dx = dx;
    for(int d = 0; d < 3; ++d) {
        h->g.boxMin[d] = P.box_min[d];
        h->g.boxMax[d] = P.box_max[d];
        h->g.bmin[d] = P.box_min[d] - pad;
        const float bmax = P.box_max[d] + pad;
        h->g.G[d] = (int)(uint32_t)std::ceil((bmax - h->g.bmin[d]) / dx);
        if(h->g.G[d] < 3) { delete h; return BNN_ERR_INVALID_ARGUMENT; }
    }
    h->g.sdfRadius = dx * (float)(1.01 * std::sqrt(3.0) / 2.0);
    h->frameDuration = P.frame_duration;
    h->frameTime = P.frame_duration;
    h->C = (size_t)h->g.G[0] * h->g.G[1] * h->g.G[2];
    if(h->C >= (size_t)0x7fffffff) { delete h; return BNN_ERR_NOT_SUPPORTED; }
    if(h->g.G[0] > 65535) {
        // the packed pressure rows store y-neighbour row distances in 16 bits
        bnn_set_error("bnn_flip_create: more than 65535 cells along x");
        delete h;
        return BNN_ERR_NOT_SUPPORTED;
    }
    for(int d = 0; d < 3; ++d) h->F[d] = (size_t)face_sx(h->g, d) * face_sy(h->g, d) * face_sz(h->g, d);
    cudaError_t e = cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking);
    if(e != cudaSuccess) { bnn_set_error(cudaGetErrorString(e)); delete h; return BNN_ERR_CUDA; }
    int rc = BNN_OK;
    auto ok = [&](cudaError_t err) {
        if(err != cudaSuccess && rc == BNN_OK) {
            bnn_set_error(cudaGetErrorString(err));
            rc = err == cudaErrorMemoryAllocation ? BNN_ERR_OUT_OF_MEMORY : BNN_ERR_CUDA;
        }
    };
    for(int d = 0; d < 3; ++d) {
        ok(dev_alloc(&h->U[d], h->F[d] * sizeof(float)));
        ok(dev_alloc(&h->B[d], h->F[d] * sizeof(float)));
        ok(dev_alloc(&h->O[d], h->F[d] * sizeof(float)));
        ok(dev_alloc(&h->VA[d], h->F[d]));
        ok(dev_alloc(&h->VB[d], h->F[d]));
    }
    ok(dev_alloc(&h->count, h->C * sizeof(uint32_t)));
    ok(dev_alloc(&h->cellStart, (h->C + 1) * sizeof(uint32_t)));
    size_t ws = scan_workspace_bytes(h->C);
    if(ws) ok(dev_alloc(&h->scanWs, ws));
    ok(dev_alloc(&h->phi, h->C * sizeof(float)));
    ok(dev_alloc(&h->flag, h->C * sizeof(uint32_t)));
    ok(dev_alloc(&h->aidx, (h->C + 1) * sizeof(uint32_t)));
    ok(dev_alloc(&h->dst, sizeof(DevState)));
    ok(pinned_state_alloc(&h->hst));
    for(auto& ev : h->ev) ok(cudaEventCreate(&ev));
    for(auto& ev : h->io) ok(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    ok(cudaStreamCreateWithFlags(&h->s2, cudaStreamNonBlocking));
    if(rc != BNN_OK) { destroy_all(h); return rc; }
    for(int d = 0; d < 3; ++d) {
        ok(cudaMemsetAsync(h->U[d], 0, h->F[d] * sizeof(float), h->s));
        ok(cudaMemsetAsync(h->O[d], 0, h->F[d] * sizeof(float), h->s));
        ok(cudaMemsetAsync(h->VA[d], 0, h->F[d], h->s));
    }
    ok(cudaMemsetAsync(h->count, 0, h->C * sizeof(uint32_t), h->s));
    ok(cudaMemsetAsync(h->phi, 0, h->C * sizeof(float), h->s));
    ok(cudaMemsetAsync(h->aidx, 0, (h->C + 1) * sizeof(uint32_t), h->s));
    ok(cudaMemsetAsync(h->dst, 0, sizeof(DevState), h->s));
    ok(cudaStreamSynchronize(h->s));
    std::memset(h->hst, 0, sizeof(DevState));
    if(rc == BNN_OK && P.max_particles) rc = reserve_particles(h, P.max_particles);
    if(rc != BNN_OK) { destroy_all(h); return rc; }
    *out = h;
    return BNN_OK;
}

// Device bytes one handle holds, from its capacities (the allocations in bnn_flip_create,
// reserve_particles, reserve_rows and pcg_reserve).
static uint64_t device_bytes(const bnn_flip* h) {
    uint64_t b = 0;
    for(int d = 0; d < 3; ++d) b += (uint64_t)h->F[d] * 14u;                       // U, B, O + 2 valid
    b += (uint64_t)h->C * 20u + 8u + scan_workspace_bytes(h->C);                   // count..aidx
    const bool affine = h->P.solver_kind == BNN_SOLVER_APIC || h->P.solver_kind == BNN_SOLVER_AFLIP;
    b += (uint64_t)h->cap * (172u + (affine ? 72u : 0u) + (h->moved ? 12u : 0u));  // particle arrays
    b += (uint64_t)h->rowCap * 44u;                                                // rows
    b += (uint64_t)h->pcg.cap * (48u + (h->pcg.x64 ? 56u : 0u)) + (uint64_t)h->pcg.nchCap * 40u;
    return b;
}

// Bytes a scene will hold (admission estimate before creating it): the grid arrays plus
// the particle arrays for n particles, with one pressure row per particle (dense fluid
// has one row per 8 particles; thin sheets and droplets approach one per particle).
extern "C" int bnn_scene_bytes_estimate(const bnn_params* params, uint32_t n, uint64_t* bytes) {
    if(!params || !bytes || !(params->cell_size > 0.f)) return BNN_ERR_INVALID_ARGUMENT;
    uint64_t G[3];
    for(int d = 0; d < 3; ++d) {
        const float dx = params->cell_size, pad = dx * (float)params->n_expand_cells;
        const float lo = params->box_min[d] - pad, hi = params->box_max[d] + pad;
        G[d] = (uint64_t)std::ceil((hi - lo) / dx);
    }
    const uint64_t C = G[0] * G[1] * G[2];
    const uint64_t F = (G[0] + 1) * G[1] * G[2] + G[0] * (G[1] + 1) * G[2] + G[0] * G[1] * (G[2] + 1);
    const bool affine = params->solver_kind == BNN_SOLVER_APIC || params->solver_kind == BNN_SOLVER_AFLIP;
    const bool fp64 = (params->pcg_mode & BNN_PCG_MODE_MASK) != BNN_PCG_FP32;
    const uint64_t rows = n < C ? n : C;
    const bool fused = params->solver_kind != BNN_SOLVER_PIC;
    *bytes = F * 14u + C * 24u + (uint64_t)n * (172u + (affine ? 72u : 0u) + (fused ? 12u : 0u)) + rows * 44u +
             (rows * 5u / 4u + 4096u) * (48u + (fp64 ? 56u : 0u));
    return BNN_OK;
}

extern "C" int bnn_flip_device_bytes(bnn_flip* h, uint64_t* bytes) {
    if(!h || !bytes) return BNN_ERR_INVALID_ARGUMENT;
    *bytes = device_bytes(h);
    return BNN_OK;
}

extern "C" int bnn_flip_destroy(bnn_flip* h) {
    if(!h) return BNN_ERR_INVALID_ARGUMENT;
    if(h->s) cudaStreamSynchronize(h->s);
    destroy_all(h);
    return BNN_OK;
}

extern "C" int bnn_flip_stream(bnn_flip* h, void** stream) {
    if(!h || !stream) return BNN_ERR_INVALID_ARGUMENT;
    *stream = (void*)h->s;
    return BNN_OK;
}

extern "C" int bnn_flip_grid_dims(bnn_flip* h, int32_t g[3]) {
    if(!h || !g) return BNN_ERR_INVALID_ARGUMENT;
    for(int d = 0; d < 3; ++d) g[d] = h->g.G[d];
    return BNN_OK;
}

extern "C" int bnn_flip_num_particles(bnn_flip* h, uint32_t* n) {
    if(!h || !n) return BNN_ERR_INVALID_ARGUMENT;
    *n = h->n;
    return BNN_OK;
}

// Upload into the current SoA buffers in caller order (ids = 0..n-1)
static int upload_particles(bnn_flip* h, const float* pos, const float* vel, uint32_t n) {
    BNN_CUDA_CHECK(cudaMemcpyAsync(h->aosStage, pos, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, h->s));
    BNN_CUDA_CHECK(cudaMemcpyAsync(h->aosStage + 3 * (size_t)h->cap, vel, 3 * (size_t)n * sizeof(float),
                                   cudaMemcpyHostToDevice, h->s));
    launch_aos_to_soa((int)n, h->aosStage, h->aosStage + 3 * (size_t)h->cap, h->p6[h->cur], h->ids[h->cur], h->cap, h->s);
    return BNN_OK;
}

extern "C" int bnn_flip_set_particles(bnn_flip* h, const float* pos, const float* vel, uint32_t n) {
    if(!h || (n && (!pos || !vel))) return BNN_ERR_INVALID_ARGUMENT;
    if((size_t)n >= (size_t)0x7fffffff) return BNN_ERR_INVALID_ARGUMENT;
    int rc = reserve_particles(h, n);
    if(rc != BNN_OK) return rc;
    h->n = n;
    h->cur = 0;
    h->premoved = false;
    if(n) {
        rc = upload_particles(h, pos, vel, n);
        if(rc != BNN_OK) return rc;
    }
    if(h->C9[0]) BNN_CUDA_CHECK(cudaMemsetAsync(h->C9[0], 0, 9 * (size_t)h->cap * sizeof(float), h->s));
    for(int d = 0; d < 3; ++d) {
        BNN_CUDA_CHECK(cudaMemsetAsync(h->U[d], 0, h->F[d] * sizeof(float), h->s));
        BNN_CUDA_CHECK(cudaMemsetAsync(h->O[d], 0, h->F[d] * sizeof(float), h->s));
        BNN_CUDA_CHECK(cudaMemsetAsync(h->VA[d], 0, h->F[d], h->s));
    }
    BNN_CUDA_CHECK(cudaMemsetAsync(h->count, 0, h->C * sizeof(uint32_t), h->s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(h->s));
    h->maxvelBits = 0;
    h->frameTime = h->frameDuration;
    h->nRows = 0;
    return BNN_OK;
}

extern "C" int bnn_flip_get_particles(bnn_flip* h, float* pos, float* vel) {
    if(!h || (h->n && (!pos || !vel))) return BNN_ERR_INVALID_ARGUMENT;
    if(!h->n) return BNN_OK;
    launch_soa_to_aos((int)h->n, h->p6[h->cur], h->ids[h->cur], h->aosStage, h->aosStage + 3 * (size_t)h->cap, h->cap,
                      h->s);
    BNN_CUDA_CHECK(cudaMemcpyAsync(pos, h->aosStage, 3 * (size_t)h->n * sizeof(float), cudaMemcpyDeviceToHost, h->s));
    BNN_CUDA_CHECK(cudaMemcpyAsync(vel, h->aosStage + 3 * (size_t)h->cap, 3 * (size_t)h->n * sizeof(float),
                                   cudaMemcpyDeviceToHost, h->s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(h->s));
    return BNN_OK;
}

extern "C" int bnn_flip_device_particles(bnn_flip* h, float** p6, uint32_t** ids) {
    if(!h) return BNN_ERR_INVALID_ARGUMENT;
    {
        const int rc = drop_premove(h);  // the caller may change the particles through these pointers
        if(rc != BNN_OK) return rc;
    }
    if(p6) *p6 = h->p6[h->cur];
    if(ids) *ids = h->ids[h->cur];
    return BNN_OK;
}

// Replace the face velocities of one component (a saved memory state, PIC_Solver::
// loadMemoryState, PIC_Solver.cpp:158-206); the CFL maximum is taken from the new field.
extern "C" int bnn_flip_set_grid(bnn_flip* h, int32_t field, const float* in, size_t count) {
    if(!h || !in || field < BNN_FIELD_U || field > BNN_FIELD_W) return BNN_ERR_INVALID_ARGUMENT;
    if(count != h->F[field]) return BNN_ERR_INVALID_ARGUMENT;
    {
        const int rc = drop_premove(h);
        if(rc != BNN_OK) return rc;
    }
    BNN_CUDA_CHECK(cudaMemcpyAsync(h->U[field], in, count * sizeof(float), cudaMemcpyHostToDevice, h->s));
    BNN_CUDA_CHECK(cudaMemsetAsync(&h->dst->maxvel_bits, 0, sizeof(unsigned), h->s));
    for(int d = 0; d < 3; ++d) launch_maxabs(h->U[d], h->F[d], &h->dst->maxvel_bits, h->s);
    BNN_CUDA_CHECK(cudaMemcpyAsync(&h->hst->maxvel_bits, &h->dst->maxvel_bits, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                   h->s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(h->s));
    h->maxvelBits = h->hst->maxvel_bits;
    return BNN_OK;
}

extern "C" int bnn_flip_get_grid(bnn_flip* h, int32_t field, float* out, size_t count) {
    if(!h || !out) return BNN_ERR_INVALID_ARGUMENT;
    const float* src = nullptr;
    size_t need = 0;
    if(field >= BNN_FIELD_U && field <= BNN_FIELD_W) { src = h->U[field]; need = h->F[field]; }
    else if(field >= BNN_FIELD_OLD_U && field <= BNN_FIELD_OLD_W) { src = h->O[field - 5]; need = h->F[field - 5]; }
    else if(field == BNN_FIELD_PHI) { src = h->phi; need = h->C; }
    else if(field >= BNN_FIELD_WEIGHT_U && field <= BNN_FIELD_WEIGHT_W) {
        // weights 1 while no dynamic boundary has been set
        const int d = field - BNN_FIELD_WEIGHT_U;
        need = h->F[d];
        if(count < need) return BNN_ERR_INVALID_ARGUMENT;
        if(!h->gridBoundary) {
            for(size_t i = 0; i < need; ++i) out[i] = 1.0f;
            return BNN_OK;
        }
        src = h->W[d];
    } else if(field == BNN_FIELD_BOUNDARY_SDF) {
        need = (size_t)(h->g.G[0] + 1) * (h->g.G[1] + 1) * (h->g.G[2] + 1);
        if(count < need) return BNN_ERR_INVALID_ARGUMENT;
        if(!h->gridBoundary) {
            // never computed for static scenes (the reference's array stays at 0)
            for(size_t i = 0; i < need; ++i) out[i] = 0.0f;
            return BNN_OK;
        }
        src = h->nodeSdf;
    }
    else if(field == BNN_FIELD_PRESSURE || field == BNN_FIELD_ACTIVE) {
        need = h->C;
        if(count < need) return BNN_ERR_INVALID_ARGUMENT;
        if(!h->cellTmp) BNN_CUDA_CHECK(dev_alloc(&h->cellTmp, h->C * sizeof(float)));
        if(h->nRows == 0 && field == BNN_FIELD_PRESSURE) {
            BNN_CUDA_CHECK(cudaMemsetAsync(h->cellTmp, 0, h->C * sizeof(float), h->s));
        } else {
            launch_cells_from_rows(h->C, h->phi, h->aidx, h->pressure, h->cellTmp, field == BNN_FIELD_ACTIVE, h->s);
        }
        src = h->cellTmp;
    } else {
        return BNN_ERR_INVALID_ARGUMENT;
    }
    if(count < need) return BNN_ERR_INVALID_ARGUMENT;
    BNN_CUDA_CHECK(cudaMemcpyAsync(out, src, need * sizeof(float), cudaMemcpyDeviceToHost, h->s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(h->s));
    return BNN_OK;
}

// ParticleSolver::generateBoundaries (ParticleSolver.cpp:242-295) for the domain box plus
// the given objects: the domain box (ParticleSolver.cpp:76-82, untransformed) and the
// static objects form one CSG union, each dynamic object stays on its own.  With a
// dynamic object and update_grid the node SDF and face weights are recomputed now; they
// then stay until the next update, like the reference's boundarySDF array.
extern "C" int bnn_flip_set_boundaries(bnn_flip* h, const bnn_boundary_object* objs, uint32_t n,
                                       int32_t update_grid) {
    if(!h || (n && !objs) || n >= (uint32_t)kMaxBoundaryObjects) return BNN_ERR_INVALID_ARGUMENT;
    {
        const int rc = drop_premove(h);  // the next move must see these objects
        if(rc != BNN_OK) return rc;
    }
    std::vector<BObj> list;
    BObj box{};
    box.geometry = 0;
    box.transformed = 0;
    box.scale = 1.0f;
    for(int d = 0; d < 3; ++d) { box.bmin[d] = h->g.boxMin[d]; box.bmax[d] = h->g.boxMax[d]; }
    list.push_back(box);
    bool anyDynamic = false;
    for(int pass = 0; pass < 2; ++pass)
        for(uint32_t i = 0; i < n; ++i) {
            const bnn_boundary_object& o = objs[i];
            if(o.geometry != BNN_GEOMETRY_BOX && o.geometry != BNN_GEOMETRY_SPHERE) return BNN_ERR_NOT_SUPPORTED;
            if((o.dynamic != 0) != (pass == 1)) continue;
            BObj b{};
            b.geometry = o.geometry;
            b.transformed = o.transformed ? 1 : 0;
            b.scale = o.uniform_scale;
            for(int d = 0; d < 3; ++d) { b.bmin[d] = o.box_min[d]; b.bmax[d] = o.box_max[d]; }
            for(int q = 0; q < 12; ++q) b.M[q] = o.inv_transform[q];
            list.push_back(b);
            anyDynamic |= pass == 1;
        }
    uint32_t nStatic = 1;
    for(uint32_t i = 0; i < n; ++i) nStatic += objs[i].dynamic ? 0u : 1u;
    if(!h->objDev) BNN_CUDA_CHECK(dev_alloc(&h->objDev, kMaxBoundaryObjects * sizeof(BObj)));
    BNN_CUDA_CHECK(cudaMemcpyAsync(h->objDev, list.data(), list.size() * sizeof(BObj), cudaMemcpyHostToDevice, h->s));
    if(n == 0) {
        h->g.obj = nullptr;
        h->g.nObj = 0;
        h->g.nStatic = 0;
    } else {
        h->g.obj = h->objDev;
        h->g.nObj = (int)list.size();
        h->g.nStatic = (int)nStatic;
    }
    if(n == 0) h->gridBoundary = false;
    if(anyDynamic && update_grid) {
        h->gridBoundary = true;
        const size_t nn = (size_t)(h->g.G[0] + 1) * (h->g.G[1] + 1) * (h->g.G[2] + 1);
        if(!h->nodeSdf) BNN_CUDA_CHECK(dev_alloc(&h->nodeSdf, nn * sizeof(float)));
        for(int d = 0; d < 3; ++d)
            if(!h->W[d]) BNN_CUDA_CHECK(dev_alloc(&h->W[d], h->F[d] * sizeof(float)));
        launch_boundary_grid(h->g, h->nodeSdf, h->W, h->s);
    }
    BNN_CUDA_CHECK(cudaGetLastError());
    BNN_CUDA_CHECK(cudaStreamSynchronize(h->s));
    return BNN_OK;
}

// Host arrays of bnn_flip_step_host whose transfers overlap the step: the main stream waits
// for the velocity upload only where the sort first gathers velocities, and the positions,
// final after the sort, go back to the host on the copy stream while the rest of the step
// runs.  Their download is issued after the step's last small device-to-host read before
// the pressure solve (the active-row count): copies in one direction share a copy engine,
// so that read would otherwise wait for the whole 12 bytes per particle to cross the link.
struct HostIo {
    bool velPending = false;  // velocities still being uploaded on s2 (event io[1])
    float* posOut = nullptr;  // host array for the final positions (caller order)
};

static int run_substep(bnn_flip* h, bnn_step_stats* st, const HostIo* io = nullptr) {
    cudaStream_t s = h->s;
    const GridDesc& g = h->g;
    const float substep = begin_substep(h);
    const float sub = substep / (float)h->P.advection_steps;
    const int kind = h->P.solver_kind;
    const bool affine = kind == BNN_SOLVER_APIC || kind == BNN_SOLVER_AFLIP;
    const int n = (int)h->n;
    // the move already ran at the end of the last sub-step: with the size computed there
    const bool moved = h->premoved && n > 0;
    if(moved && substep != h->premovedDt) {
        drop_premove(h);
        bnn_set_error("sub-step size of the fused move differs from the host's");
        return BNN_ERR_DEVICE_CHECK;
    }
    h->premoved = false;

    cudaEventRecord(h->ev[0], s);
    if(moved) {
        launch_step_reset_moved(h->dst, s);
    } else {
        launch_step_reset(h->dst, s);
        // moveParticles + counting sort (histogram while advecting)
        launch_advect(n, h->p6[h->cur], h->cap, h->U, g, sub, (int)h->P.advection_steps, h->cellOf, h->slot, h->count,
                      h->dst, h->bboxPart, s);
    }
    cudaEventRecord(h->ev[1], s);
    BNN_CUDA_CHECK(exclusive_scan_u32(h->count, h->cellStart, h->C, h->scanWs, s));
    const int nxt = 1 - h->cur;
    // the particles' gather is the first reader of the velocities: it alone waits for
    // their upload (bnn_flip_step_host)
    launch_sort_finish(n, h->C, h->cellOf, h->slot, h->cellStart, h->order, h->key, h->count, h->p6[h->cur],
                       moved ? h->moved : nullptr, h->p6[nxt],
                       h->ids[h->cur], h->ids[nxt], affine ? h->C9[h->cur] : nullptr, affine ? h->C9[nxt] : nullptr,
                       h->rec, g, h->cap, h->dst, s, io && io->velPending ? h->io[1] : nullptr);
    h->cur = nxt;
    if(h->P.correct_position && n > 0) {
        // PIC_Solver::advanceFrame: correctParticlePositions right after moveParticles
        // (PIC_Solver.cpp:292-293), on the sorted particles; then they are binned again
        const float pr = h->P.cell_size / h->P.ratio_cell_size_p_radius;
        const float radius = 2.0f * pr / (float)std::sqrt(3.0);
        const float threshold = 0.01f * radius;
        const float kSpring = radius * sub * h->P.repulsive_force_stiffness;
        launch_correct_positions(n, g, h->p6[h->cur], h->cap, h->ids[h->cur], h->cellStart, radius * radius,
                                 threshold * threshold, threshold / substep, kSpring, (int)h->P.advection_steps,
                                 h->substepIndex, h->aosStage, s);
        BNN_CUDA_CHECK(cudaMemcpyAsync(h->p6[h->cur], h->aosStage, 3 * (size_t)h->cap * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s));
        launch_rebin(n, h->p6[h->cur], h->cap, g, h->cellOf, h->slot, h->count, h->dst, s);
        BNN_CUDA_CHECK(exclusive_scan_u32(h->count, h->cellStart, h->C, h->scanWs, s));
        const int nxt2 = 1 - h->cur;
        launch_sort_finish(n, h->C, h->cellOf, h->slot, h->cellStart, h->order, h->key, h->count, h->p6[h->cur], nullptr, h->p6[nxt2],
                           h->ids[h->cur], h->ids[nxt2], affine ? h->C9[h->cur] : nullptr,
                           affine ? h->C9[nxt2] : nullptr, h->rec, g, h->cap, h->dst, s);
        h->cur = nxt2;
    }
    cudaEventRecord(h->ev[2], s);
    if(io && io->posOut && n > 0) {
        // positions are final from here on (the rest of the step reads them only): back
        // to the caller's order and to the host on the copy stream
        BNN_CUDA_CHECK(cudaEventRecord(h->io[2], s));
        BNN_CUDA_CHECK(cudaStreamWaitEvent(h->s2, h->io[2], 0));
        launch_soa3_to_aos(n, h->p6[h->cur], h->ids[h->cur], h->aosStage, h->cap, h->s2);
    }
    // P2G
    if(kind == BNN_SOLVER_PIC) {
        // PIC_Solver::advanceVelocity (PIC_Solver.cpp:332-338): the grid velocity is advected
        launch_advect_grid(g, h->U, h->B, substep, s);
    } else if(affine) {
        // APIC / AFLIP: the same pass with the affine momentum term
        launch_p2g_sdf_affine(g, h->dst, h->cellStart, h->rec, h->C9[h->cur], h->cap, h->U, h->VA, h->phi, s);
    } else {
        // FLIP: the three components and the fluid SDF in one pass over the particles (the
        // SDF reads positions only, so it is final here already)
        launch_p2g_sdf(g, h->dst, h->cellStart, h->rec, h->cap, h->U, h->VA, h->phi, s);
    }
    cudaEventRecord(h->ev[3], s);
    const float gdt = h->P.apply_gravity ? 9.81f * substep : 0.f;
    if(kind == BNN_SOLVER_APIC || kind == BNN_SOLVER_PIC) {
        // APIC_Solver::advanceVelocity: P2G then gravity, no extrapolation / backup; PIC:
        // advection then gravity
        if(h->P.apply_gravity) launch_add_scalar(h->U[1], h->F[1], -gdt, s);
    } else {
        // extrapolate, backup oldVels, Earth gravity (FLIP_Solver.cpp:44-47)
        if(h->gridBoundary) {
            // ... with constrainGridVelocity between the extrapolation and the backup
            launch_extrapolate(g, h->U, h->VA, h->B, h->VB, 0, nullptr, 0.f, h->dst, s);
            launch_constrain_velocity(g, h->dst, h->U, h->VA, h->W, h->nodeSdf, h->B, s);
            for(int d = 0; d < 3; ++d)
                BNN_CUDA_CHECK(cudaMemcpyAsync(h->O[d], h->U[d], h->F[d] * sizeof(float), cudaMemcpyDeviceToDevice, s));
            if(h->P.apply_gravity) launch_add_scalar(h->U[1], h->F[1], -gdt, s);
        } else {
            launch_extrapolate(g, h->U, h->VA, h->B, h->VB, 1, h->O, gdt, h->dst, s);
        }
    }
    cudaEventRecord(h->ev[4], s);
    // pressure projection (PIC_Solver.cpp:533-539)
    if(kind == BNN_SOLVER_PIC) launch_fluid_sdf_tile(g, h->dst, h->cellStart, h->rec, h->cap, h->phi, s);
    if(h->gridBoundary) launch_solid_extend(g, h->nodeSdf, h->phi, s);
    cudaEventRecord(h->ev[5], s);
    launch_active_flags(g, h->phi, h->flag, h->dst, s);
    BNN_CUDA_CHECK(exclusive_scan_u32(h->flag, h->aidx, h->C, h->scanWs, s));
    uint32_t nrows = 0;
    BNN_CUDA_CHECK(cudaMemcpyAsync(&h->hst->n_active, h->aidx + h->C, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    nrows = h->hst->n_active;
    if(io && io->posOut && n > 0)
        BNN_CUDA_CHECK(cudaMemcpyAsync(io->posOut, h->aosStage, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost,
                                       h->s2));
    int rc = reserve_rows(h, nrows);
    if(rc != BNN_OK) return rc;
    h->nRows = nrows;
    launch_active_rows(h->C, h->flag, h->aidx, h->rowCell, s);
    if(h->gridBoundary && h->coefCap < h->rowCap) {
        dev_free(h->coef);
        h->coef = nullptr;
        h->coefCap = 0;
        BNN_CUDA_CHECK(dev_alloc(&h->coef, 6 * (size_t)h->rowCap * sizeof(float)));
        h->coefCap = h->rowCap;
    }
    launch_build_rows(g, (int)nrows, h->rowCell, h->phi, h->aidx, h->U, h->gridBoundary ? h->W : nullptr, substep,
                      h->rhs, h->diag, h->invd, h->nbr, h->gridBoundary ? h->coef : nullptr, h->dst, s);
    cudaEventRecord(h->ev[6], s);
    PcgOutcome po;
    rc = pcg_solve(h->pcg, (int)nrows, h->rhs, h->diag, h->invd, h->nbr, h->gridBoundary ? h->coef : nullptr,
                   true, substep, h->P.pcg_mode,
                   h->P.cg_relative_tolerance, h->P.max_cg_iteration, h->P.refine_inner_tolerance,
                   h->P.refine_tolerance, h->pressure, nullptr, h->dst, h->hst, s, po);
    if(rc != BNN_OK) return rc;
    cudaEventRecord(h->ev[7], s);
    // projected faces go to the ping-pong arrays, which then become the velocity arrays
    launch_update_velocity(g, h->dst, h->phi, h->aidx, h->pressure, substep, h->U, h->B, h->VB,
                           h->gridBoundary ? h->W : nullptr, s);
    launch_extrapolate(g, h->B, h->VB, h->U, h->VA, h->gridBoundary ? 0 : 2, nullptr, 0.f, h->dst, s);
    for(int d = 0; d < 3; ++d) {
        std::swap(h->U[d], h->B[d]);
        std::swap(h->VA[d], h->VB[d]);
    }
    if(h->gridBoundary) {
        // constrainGridVelocity after the extrapolation (FLIP_Solver.cpp:51), then the CFL
        // maximum over the constrained faces
        launch_constrain_velocity(g, h->dst, h->U, h->VA, h->W, h->nodeSdf, h->B, s);
        for(int d = 0; d < 3; ++d) launch_maxabs(h->U[d], h->F[d], &h->dst->maxvel_bits, s);
    }
    cudaEventRecord(h->ev[8], s);
    // PIC_Solver leaves the particle velocities alone (no grid-to-particle transfer).  FLIP,
    // APIC and AFLIP steps driven from device-resident particles also move the particles for
    // the next sub-step here (k_g2p_move); a step on caller arrays (bnn_flip_step_host) does
    // not, since the next call brings new particle data, and neither does a scene with
    // dynamic boundary objects, which are moved (bnn_flip_set_boundaries) before every
    // sub-step.
    const bool fuse = kind != BNN_SOLVER_PIC && n > 0 && !io && h->moved && !h->gridBoundary;
    if(fuse) {
        NextStep ns;
        ns.frameTime = h->frameTime + substep;
        ns.frameDuration = h->frameDuration;
        ns.cfl = h->P.cfl_factor;
        ns.minDt = h->P.min_timestep;
        ns.maxDt = h->P.max_timestep;
        ns.advSteps = (int)h->P.advection_steps;
        launch_g2p_move(n, g, h->p6[h->cur], h->cap, h->U, h->O, h->P.pic_flip_ratio, kind,
                        affine ? h->C9[h->cur] : nullptr, ns, h->moved, h->cellOf, h->slot,
                        h->count, h->dst, h->bboxPart, s);
    } else if(kind != BNN_SOLVER_PIC) {
        launch_g2p(n, g, h->p6[h->cur], h->cap, h->U, h->O, h->P.pic_flip_ratio, kind, affine ? h->C9[h->cur] : nullptr,
                   s);
    }
    cudaEventRecord(h->ev[9], s);
    BNN_CUDA_CHECK(cudaGetLastError());
    BNN_CUDA_CHECK(cudaMemcpyAsync(h->hst, h->dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    h->maxvelBits = h->hst->maxvel_bits;
    h->frameTime += substep;
    ++h->substepIndex;
    if(fuse) {
        h->premoved = true;
        h->premovedDt = h->hst->next_dt;
    }
    if(st) {
        st->dt = substep;
        st->frame_time = h->frameTime;
        st->frame_finished = h->frameTime >= h->frameDuration ? 1u : 0u;
        st->pcg_iterations = po.iterations;
        st->pcg_residual = po.residual;
        st->pcg_success = po.success;
        st->n_active = nrows;
        st->outer_iterations = po.outer;
        st->pcg_kernel_ms = po.kernelMs;
        st->zero_phi_cells = h->hst->zero_phi;
        st->device_flags = h->hst->flags;
        const int map[10][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {7, 8}, {8, 9}, {0, 9}};
        for(int q = 0; q < 10; ++q) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, h->ev[map[q][0]], h->ev[map[q][1]]);
            st->stage_ms[q] = ms;
        }
    }
    if(h->hst->flags & BNN_FLAG_OUT_OF_GRID) return BNN_ERR_DEVICE_CHECK;
    if(!po.success) return BNN_ERR_PCG_NOT_CONVERGED;
    return BNN_OK;
}

extern "C" int bnn_flip_step(bnn_flip* h, bnn_step_stats* st) {
    if(!h) return BNN_ERR_INVALID_ARGUMENT;
    if(st) std::memset(st, 0, sizeof(*st));
    return run_substep(h, st);
}

// The caller's arrays are in caller order (the order bnn_flip_get_particles returns): the
// ids restart at 0..n-1 and the device-only per-particle data (APIC / AFLIP affine
// matrices) is brought into that order.  The sort is by (cell, id), so the step computes
// the same result as the resident path.  Positions go up
// first on the main stream (the move needs them); velocities go up on the copy stream
// while the particles move and are binned; the final positions come back on the copy
// stream while the grid work runs, and the velocities after the grid-to-particle
// transfer.
extern "C" int bnn_flip_step_host(bnn_flip* h, float* pos, float* vel, bnn_step_stats* st) {
    if(!h || (h->n && (!pos || !vel))) return BNN_ERR_INVALID_ARGUMENT;
    if(st) std::memset(st, 0, sizeof(*st));
    const int n = (int)h->n;
    const size_t cap = h->cap;
    HostIo io;
    {
        const int rc = drop_premove(h);  // new particle data from the caller
        if(rc != BNN_OK) return rc;
    }
    if(n) {
        cudaStream_t s = h->s, s2 = h->s2;
        if(h->C9[h->cur]) {
            // the affine matrices (APIC / AFLIP) stay on the device: bring them into the
            // caller's order, the order the ids restart in
            launch_scatter_planes(n, 9, h->C9[h->cur], h->ids[h->cur], h->C9[1 - h->cur], cap, s);
            std::swap(h->C9[0], h->C9[1]);
        }
        // positions first and alone on the link (the advection needs them), then the
        // velocities, which the step needs only from the sort's gather on
        BNN_CUDA_CHECK(cudaMemcpyAsync(h->aosStage, pos, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s));
        BNN_CUDA_CHECK(cudaEventRecord(h->io[0], s));
        BNN_CUDA_CHECK(cudaStreamWaitEvent(s2, h->io[0], 0));
        launch_aos3_to_soa(n, h->aosStage, h->p6[h->cur], h->ids[h->cur], cap, s);
        BNN_CUDA_CHECK(cudaMemcpyAsync(h->aosStage + 3 * cap, vel, 3 * (size_t)n * sizeof(float),
                                       cudaMemcpyHostToDevice, s2));
        launch_aos3_to_soa(n, h->aosStage + 3 * cap, h->p6[h->cur] + 3 * cap, nullptr, cap, s2);
        BNN_CUDA_CHECK(cudaEventRecord(h->io[1], s2));
        io.velPending = true;
        io.posOut = pos;
    }
    int rc = run_substep(h, st, &io);
    if(n) {
        cudaStream_t s = h->s;
        if(rc == BNN_OK || rc == BNN_ERR_PCG_NOT_CONVERGED || rc == BNN_ERR_DEVICE_CHECK) {
            launch_soa3_to_aos(n, h->p6[h->cur] + 3 * cap, h->ids[h->cur], h->aosStage + 3 * cap, cap, s);
            cudaError_t e = cudaMemcpyAsync(vel, h->aosStage + 3 * cap, 3 * (size_t)n * sizeof(float),
                                            cudaMemcpyDeviceToHost, s);
            if(e != cudaSuccess && rc == BNN_OK) { bnn_set_error(cudaGetErrorString(e)); rc = BNN_ERR_CUDA; }
        }
        cudaError_t e1 = cudaStreamSynchronize(h->s2);
        cudaError_t e2 = cudaStreamSynchronize(s);
        if((e1 != cudaSuccess || e2 != cudaSuccess) && rc == BNN_OK) {
            bnn_set_error(cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            rc = BNN_ERR_CUDA;
        }
    }
    return rc;
}

// AnisotropicKernelGenerator over the solver's particles (PIC_Solver::saveFrameData,
// PIC_Solver.cpp:248-252, constructs it with the particle positions and
// solverParams().particleRadius).  The particles are binned and sorted first, the same
// sort every sub-step starts from, so the pass works on any state (also before the first
// step); the order it leaves them in does not change any later result, because each
// sub-step sorts by (cell, id) again.
extern "C" int bnn_flip_anisotropic_kernels(bnn_flip* h, const bnn_aniso_params* params, float* centers,
                                            float* matrices, bnn_aniso_stats* stats) {
    if(!h || (h->n && (!centers || !matrices))) return BNN_ERR_INVALID_ARGUMENT;
    bnn_aniso_params prm = params ? *params : aniso_defaults(0.0f);
    if(!(prm.particle_radius > 0.0f)) prm.particle_radius = h->P.cell_size / h->P.ratio_cell_size_p_radius;
    int rc = aniso_check_params(prm);
    if(rc != BNN_OK) return rc;
    if(stats) std::memset(stats, 0, sizeof(*stats));
    const int n = (int)h->n;
    const GridDesc& g = h->g;
    if(stats) {
        for(int d = 0; d < 3; ++d) { stats->grid_bmin[d] = g.bmin[d]; stats->grid_dims[d] = g.G[d]; }
        stats->grid_cell_size = g.dx;
    }
    if(n == 0) return BNN_OK;
    cudaStream_t s = h->s;
    const bool affine = h->P.solver_kind == BNN_SOLVER_APIC || h->P.solver_kind == BNN_SOLVER_AFLIP;
    rc = drop_premove(h);  // the re-sort below reuses the move's buffers
    if(rc != BNN_OK) return rc;
    launch_rebin(n, h->p6[h->cur], h->cap, g, h->cellOf, h->slot, h->count, h->dst, s);
    BNN_CUDA_CHECK(exclusive_scan_u32(h->count, h->cellStart, h->C, h->scanWs, s));
    const int nxt = 1 - h->cur;
    launch_sort_finish(n, h->C, h->cellOf, h->slot, h->cellStart, h->order, h->key, h->count, h->p6[h->cur], nullptr, h->p6[nxt],
                       h->ids[h->cur], h->ids[nxt], affine ? h->C9[h->cur] : nullptr, affine ? h->C9[nxt] : nullptr,
                       h->rec, g, h->cap, h->dst, s);
    h->cur = nxt;
    const size_t cap = h->cap;
    if(!h->aniso) BNN_CUDA_CHECK(dev_alloc(&h->aniso, (12 * cap + 4) * sizeof(float)));
    float* dC = h->aniso;
    float* dM = h->aniso + 3 * cap;
    unsigned* cnt = (unsigned*)(h->aniso + 12 * cap);
    BNN_CUDA_CHECK(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), s));
    AnisoGrid ag;
    for(int d = 0; d < 3; ++d) { ag.G[d] = g.G[d]; ag.bmin[d] = g.bmin[d]; }
    ag.dx = g.dx;
    cudaEventRecord(h->ev[0], s);
    launch_aniso(n, h->rec + 3 * cap, h->ids[h->cur], h->cellStart, ag, prm, dC, dM, cnt, s);
    cudaEventRecord(h->ev[1], s);
    BNN_CUDA_CHECK(cudaMemcpyAsync(centers, dC, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaMemcpyAsync(matrices, dM, 9 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s));
    unsigned hc[2] = {0u, 0u};
    BNN_CUDA_CHECK(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    BNN_CUDA_CHECK(cudaGetLastError());
    if(stats) {
        stats->sprays = hc[0];
        cudaEventElapsedTime(&stats->ms, h->ev[0], h->ev[1]);
    }
    if(hc[1]) {
        bnn_set_error("bnn_flip_anisotropic_kernels: a particle lies outside the grid");
        return BNN_ERR_DEVICE_CHECK;
    }
    return BNN_OK;
}

extern "C" int bnn_flip_advance_frame(bnn_flip* h, uint32_t* substeps) {
    if(!h) return BNN_ERR_INVALID_ARGUMENT;
    uint32_t k = 0;
    bnn_step_stats st;
    do {
        int rc = bnn_flip_step(h, &st);
        ++k;
        if(rc != BNN_OK) { if(substeps) *substeps = k; return rc; }
    } while(!st.frame_finished);
    if(substeps) *substeps = k;
    return BNN_OK;
}

// ---------------------------------------------------------------------------------
// Standalone PCG on a 7-point system
// ---------------------------------------------------------------------------------
namespace bnn {
std::string tile_tuning_report();
}
extern "C" int bnn_tile_shapes(int32_t* tz, int32_t* yc, int32_t cap) {
    for(int k = 0; k < kTileShapes && k < cap; ++k) {
        int a = 0, b = 0;
        tile_shape_dims(k, &a, &b);
        if(tz) tz[k] = a;
        if(yc) yc[k] = b;
    }
    return kTileShapes;
}
extern "C" int bnn_set_tile_shape(int32_t shape) { return tile_shape_set(shape); }
extern "C" int bnn_tile_tuning(char* buf, size_t cap, size_t* needed) {
    const std::string r = tile_tuning_report();
    if(needed) *needed = r.size() + 1;
    if(!buf || cap < r.size() + 1) return BNN_ERR_CAPACITY;
    std::memcpy(buf, r.c_str(), r.size() + 1);
    return BNN_OK;
}

extern "C" int bnn_pcg_barrier_probe(float limit_seconds, int32_t* barrier_status, float* elapsed_ms) {
    if(!barrier_status || !elapsed_ms || !(limit_seconds > 0.f && limit_seconds <= 10.f)) return BNN_ERR_INVALID_ARGUMENT;
    int st = BNN_OK;
    float ms = 0.f;
    const int rc = bnn::pcg_barrier_probe(limit_seconds, &st, &ms);
    if(rc != BNN_OK) return rc;
    *barrier_status = st;
    *elapsed_ms = ms;
    return BNN_OK;
}

extern "C" int bnn_pcg_solve_7pt(uint32_t n, const float* diag, const int32_t* nbr, float offdiag, const float* rhs,
                                 float tol, uint32_t max_iter, int32_t mode, float inner_tol, double* x_out,
                                 bnn_pcg_stats* stats) {
    if(!diag || !nbr || !rhs || !x_out || (mode & ~(BNN_PCG_MODE_MASK | BNN_PCG_SINGLE_REDUCTION)) != 0 ||
       (mode & BNN_PCG_MODE_MASK) > 2)
        return BNN_ERR_INVALID_ARGUMENT;
    if(!(offdiag <= 0.f)) return BNN_ERR_INVALID_ARGUMENT;
    cudaStream_t s;
    BNN_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    float *dDiag = nullptr, *dInv = nullptr, *dRhs = nullptr, *dP = nullptr;
    int32_t* dNbr = nullptr;
    double* dX = nullptr;
    DevState *dst = nullptr, *hst = nullptr;
    PcgWork w;
    int rc = BNN_OK;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> inv(n);
    std::vector<int32_t> planes(6 * (size_t)n);
    // rows of a grid in cell order (x neighbours r-1 / r+1, y neighbours within 65535 rows,
    // z neighbours on their side) take the packed-record solve
    bool gridRows = true;
    for(uint32_t r = 0; r < n; ++r) {
        inv[r] = diag[r] != 0.f ? 1.0f / diag[r] : 0.f;
        for(int q = 0; q < 6; ++q) {
            const int32_t v = nbr[6 * (size_t)r + q];
            if(v < -1 || (v >= 0 && (uint32_t)v >= n)) {
                bnn_set_error("bnn_pcg_solve_7pt: neighbour index outside [-1, n)");
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                cudaStreamDestroy(s);
                return BNN_ERR_INVALID_ARGUMENT;
            }
            planes[(size_t)q * n + r] = v;
        }
        const int64_t R = r;
        const int32_t* nb = nbr + 6 * (size_t)r;
        if(nb[2] >= 0 && nb[2] != R - 1) gridRows = false;
        if(nb[3] >= 0 && nb[3] != R + 1) gridRows = false;
        if(nb[1] >= 0 && !(nb[1] < R && R - nb[1] <= 65535)) gridRows = false;
        if(nb[4] >= 0 && !(nb[4] > R && nb[4] - R <= 65535)) gridRows = false;
        if(nb[0] >= 0 && !(nb[0] < R)) gridRows = false;
        if(nb[5] >= 0 && !(nb[5] > R)) gridRows = false;
    }
    // the system stores -dt as the off-diagonal; recover dt so the kernels form -(1*dt)
    const float dt = -offdiag;
    size_t nn = n ? n : 1;
    auto chk = [&](cudaError_t e) { if(e != cudaSuccess && rc == BNN_OK) { bnn_set_error(cudaGetErrorString(e)); rc = BNN_ERR_CUDA; } };
    chk(cudaMalloc(&dDiag, nn * 4)); chk(cudaMalloc(&dInv, nn * 4)); chk(cudaMalloc(&dRhs, nn * 4));
    chk(cudaMalloc(&dP, nn * 4)); chk(cudaMalloc(&dNbr, 6 * nn * 4)); chk(cudaMalloc(&dX, nn * 8));
    chk(cudaMalloc(&dst, sizeof(DevState))); chk(cudaHostAlloc(&hst, sizeof(DevState), cudaHostAllocDefault));
    if(rc == BNN_OK && n) {
        chk(cudaMemcpyAsync(dDiag, diag, n * 4, cudaMemcpyHostToDevice, s));
        chk(cudaMemcpyAsync(dInv, inv.data(), n * 4, cudaMemcpyHostToDevice, s));
        chk(cudaMemcpyAsync(dRhs, rhs, n * 4, cudaMemcpyHostToDevice, s));
        chk(cudaMemcpyAsync(dNbr, planes.data(), 6 * (size_t)n * 4, cudaMemcpyHostToDevice, s));
    }
    if(rc == BNN_OK) chk(cudaMemsetAsync(dst, 0, sizeof(DevState), s));
    if(rc == BNN_OK) chk(cudaStreamSynchronize(s));
    PcgOutcome po;
    if(rc == BNN_OK) rc = pcg_reserve(w, (int)n, (mode & BNN_PCG_MODE_MASK) != BNN_PCG_FP32);  // outside the timed region
    if(rc == BNN_OK) {
        cudaEventRecord(e0, s);
        rc = pcg_solve(w, (int)n, dRhs, dDiag, dInv, dNbr, nullptr, gridRows, dt, mode, tol, max_iter, inner_tol, tol, dP, dX,
                       dst, hst, s, po);
        cudaEventRecord(e1, s);
    }
    if(rc == BNN_OK && n) chk(cudaMemcpyAsync(x_out, dX, n * 8, cudaMemcpyDeviceToHost, s));
    if(rc == BNN_OK) chk(cudaStreamSynchronize(s));
    if(stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = po.iterations;
        stats->outer_iterations = po.outer;
        stats->residual = po.residual;
        stats->success = po.success;
        float ms = 0.f;
        if(rc == BNN_OK) cudaEventElapsedTime(&ms, e0, e1);
        stats->ms = ms;
    }
    pcg_release(w);
    cudaFree(dDiag); cudaFree(dInv); cudaFree(dRhs); cudaFree(dP); cudaFree(dNbr); cudaFree(dX); cudaFree(dst);
    if(hst) cudaFreeHost(hst);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if(rc == BNN_OK && !po.success) return BNN_ERR_PCG_NOT_CONVERGED;
    return rc;
}
