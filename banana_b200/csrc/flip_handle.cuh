// The solver handle behind the C ABI's opaque bnn_flip: device state of one scene.  Shared
// by capi.cu (one scene stepped on its own stream) and batch_step.cu (many scenes stepped
// together, one launch per stage).
#pragma once

#include "bnn_internal.cuh"

#include <cfloat>
#include <cstring>

using bnn::BObj;
using bnn::DevState;
using bnn::GridDesc;
using bnn::PcgWork;

struct bnn_flip {
    bnn_params P{};
    GridDesc g{};
    size_t C = 0;      // cells
    size_t F[3] = {};  // faces per component
    float frameDuration = 0.f, frameTime = 0.f;
    uint32_t n = 0, cap = 0;
    cudaStream_t s = nullptr;
    // particles: SoA (x,y,z,vx,vy,vz) with stride cap; ping-pong for the sort
    float* p6[2] = {nullptr, nullptr};
    uint32_t* ids[2] = {nullptr, nullptr};
    float* C9[2] = {nullptr, nullptr};
    int cur = 0;
    float4* rec = nullptr;  // per-particle gather records: 3 P2G stencil planes + positions
    uint32_t *cellOf = nullptr, *slot = nullptr, *order = nullptr, *key = nullptr;
    int* bboxPart = nullptr;  // per-block occupied-cell boxes of the advection
    uint32_t *count = nullptr, *cellStart = nullptr;
    void* scanWs = nullptr;
    float* aosStage = nullptr;
    float* aniso = nullptr;  // anisotropic-kernel output: centres 3 cap, matrices 9 cap, 2 counters
    // boundary objects beyond the domain box (g.obj points at objDev)
    BObj* objDev = nullptr;
    bool gridBoundary = false;  // a dynamic object exists: node SDF, weights, constraint
    float* nodeSdf = nullptr;   // (G+1)^3
    float* W[3] = {};           // face weights
    float* coef = nullptr;      // off-diagonal values of the rows (6 planes, coefCap rows)
    int coefCap = 0;
    // faces
    float* U[3] = {};
    float* B[3] = {};
    float* O[3] = {};
    uint8_t* VA[3] = {};
    uint8_t* VB[3] = {};
    // cells
    float* phi = nullptr;
    uint32_t* flag = nullptr;
    uint32_t* aidx = nullptr; // C+1
    float* cellTmp = nullptr;
    // rows
    int rowCap = 0;
    uint32_t nRows = 0;
    uint32_t* rowCell = nullptr;
    float *rhs = nullptr, *diag = nullptr, *invd = nullptr, *pressure = nullptr;
    int32_t* nbr = nullptr;
    PcgWork pcg;
    DevState* dst = nullptr;
    DevState* hst = nullptr;
    cudaEvent_t ev[11] = {};
    // host transfers of bnn_flip_step_host that overlap the step: a copy stream and its
    // events (stream idle, velocities on the device, positions final)
    cudaStream_t s2 = nullptr;
    cudaEvent_t io[3] = {};
    unsigned maxvelBits = 0; // max|u| of the current grid (for the next CFL)
    unsigned long long substepIndex = 0;  // sub-steps taken (keys the position-correction jitter)
    // FLIP: the next sub-step's particle move runs at the end of this one (k_g2p_move); its
    // positions, cell ids, histogram and occupied-cell box then wait for the next sub-step,
    // which must use premovedDt as its size.  Anything that changes the particles, the grid
    // velocities or the boundaries in between drops it (the next sub-step moves as usual).
    float* moved = nullptr;  // 3 planes, stride cap
    bool premoved = false;
    float premovedDt = 0.f;
};

// Drops a move that ran at the end of the last sub-step (k_g2p_move) before it was used:
// its counts are still in the cell histogram, which the next binning adds to, so they
// are cleared.
inline int drop_premove(bnn_flip* h) {
    if(!h->premoved) return BNN_OK;
    h->premoved = false;
    BNN_CUDA_CHECK(cudaMemsetAsync(h->count, 0, h->C * sizeof(uint32_t), h->s));
    return BNN_OK;
}

inline int reserve_rows(bnn_flip* h, uint32_t n) {
    if((int)n <= h->rowCap) return BNN_OK;
    dev_free(h->rowCell); dev_free(h->rhs); dev_free(h->diag); dev_free(h->invd); dev_free(h->pressure); dev_free(h->nbr);
    int cap = (int)(n * 1.25) + 1024;
    if((size_t)cap > h->C) cap = (int)h->C;
    BNN_CUDA_CHECK(dev_alloc(&h->rowCell, cap * sizeof(uint32_t)));
    BNN_CUDA_CHECK(dev_alloc(&h->rhs, cap * sizeof(float)));
    BNN_CUDA_CHECK(dev_alloc(&h->diag, cap * sizeof(float)));
    BNN_CUDA_CHECK(dev_alloc(&h->invd, cap * sizeof(float)));
    BNN_CUDA_CHECK(dev_alloc(&h->pressure, cap * sizeof(float)));
    BNN_CUDA_CHECK(dev_alloc(&h->nbr, 6 * (size_t)cap * sizeof(int32_t)));
    h->rowCap = cap;
    return BNN_OK;
}

// PIC_Solver::timestepCFL (PIC_Solver.cpp:342-349) from max|u| of the current grid
inline float timestep_cfl(const bnn_flip* h) {
    float m;
    std::memcpy(&m, &h->maxvelBits, 4);
    float maxVel = FLT_MIN;
    maxVel = (maxVel < m) ? m : maxVel;
    float ts = maxVel > FLT_MIN ? h->P.cfl_factor * (h->g.dx / maxVel) : FLT_MAX;
    if(ts < h->P.min_timestep) return h->P.min_timestep;
    if(ts > h->P.max_timestep) return h->P.max_timestep;
    return ts;
}

// Starts a sub-step: wraps the frame clock and returns the sub-step size
// (PIC_Solver::advanceFrame, PIC_Solver.cpp:284-290)
inline float begin_substep(bnn_flip* h) {
    if(h->frameTime >= h->frameDuration) h->frameTime = 0.f;
    float substep = timestep_cfl(h);
    const float remaining = h->frameDuration - h->frameTime;
    if(h->frameTime + substep >= h->frameDuration) substep = remaining;
    else if(h->frameTime + 1.5f * substep >= h->frameDuration) substep = remaining * 0.5f;
    return substep;
}
