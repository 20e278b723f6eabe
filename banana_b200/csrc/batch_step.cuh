// The batched FLIP sub-step (batch_step.cu): one launch per stage over many scenes.
#pragma once

#include "flip_handle.cuh"

#include <vector>

// One captured segment of the staged step: replayed while the launch shapes it was
// captured with (sig) stay the same
struct StagedGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> sig;
    long long kernels = 0;     // kernel launches the segment holds
    // new captures so far: built into a new executable graph / written into the existing
    // one (same launches, other shapes or arguments: cudaGraphExecUpdate)
    unsigned long long instantiated = 0, updated = 0;
};

// Device tables, pinned mirror and stream of the batched step, kept between steps
struct BatchStepWork {
    bool graphs = true;        // capture the fixed segments of the step in CUDA graphs
    StagedGraph seg[2];        // before the pressure-row count, after the pressure solve
    int cap = 0;               // scenes the tables hold
    void* dev = nullptr;
    void* host = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev[10] = {};   // stage boundaries (the lone step's bnn_step_stats::stage_ms)
    bnn::BatchPcgCtx pcg;
};

// Whether the batched step takes this scene (FLIP, refined PCG in its default step order,
// the domain box as the only boundary, no position correction, particles present)
bool batch_step_eligible(const bnn_flip* h);
// One sub-step of the ns scenes hs[] (all eligible): rc[i] and st[i] are what
// bnn_flip_step would return for hs[i] alone.  Returns BNN_OK unless the batch itself
// failed (a CUDA error, a barrier timeout), which leaves the scenes' state undefined.
int batch_substep(BatchStepWork& w, bnn_flip* const* hs, int ns, int* rc, bnn_step_stats* st);
void batch_step_release(BatchStepWork& w);
