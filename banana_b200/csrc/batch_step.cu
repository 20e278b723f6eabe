// One FLIP sub-step of many scenes with one launch per stage over all of them.
//
// A scene is a full solver handle (bnn_flip); this file runs the sub-step run_substep runs
// for it (PIC_Solver::advanceFrame's body, PIC_Solver.cpp:277-305, with
// FLIP_Solver::advanceVelocity, FLIP_Solver.cpp:42-53), but each stage is one kernel launch
// whose blocks are shared out among the scenes: a per-scene block prefix tells every block
// its scene and its place in that scene's share (seg_blk), and the block runs the lone
// kernel's body on that scene's arrays.  Per-scene reductions (occupied-cell boxes, CFL
// maxima, the PCG's canonical chunk sums) stay inside the scene, so every scene computes
// bit for bit what bnn_flip_step computes for it alone.
//
// The host keeps what run_substep keeps per scene (frame clock, sub-step size, the fused
// move's size, ping-pong buffers) and reads the device only where run_substep does: the
// pressure-row counts (to size the rows) and the per-scene state at the end of the step.
// The refined pressure solves of all scenes run through pcg_solve_batch_refined.
//
// Scenes it takes (batch_step_eligible): FLIP with the refined PCG in its default step
// order, the domain box as the only boundary, no position correction, particles present.
// Everything else is stepped by bnn_flip_step on its own stream (batch.cu).
#include "flip_handle.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "batch_step.cuh"

using namespace bnn;

namespace {

constexpr unsigned kRegionBlocks = 148u * 8u;  // the lone region kernels' grid

inline unsigned cdiv(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Blocks of the lone bbox fold over the per-block boxes of a particle pass
inline unsigned bbox_fold_blocks(int n) {
    const unsigned blocks = cdiv((size_t)n, 256);
    return blocks < 148u * 4u * 256u ? (blocks + 255u) / 256u : 148u * 4u;
}

// Upper bound of the tiles (8 rows of one plane) of the extrapolation / update regions of
// component d: the whole face array
inline unsigned region_tiles(const GridDesc& g, int d) {
    const int sy = g.G[1] + (d == 1 ? 1 : 0), sz = g.G[2] + (d == 2 ? 1 : 0);
    return cdiv((size_t)sy, 8) * (unsigned)sz;
}
// The stage touches only the faces within reach of the occupied-cell box (a part of the
// array), and every block of a batched launch pays for finding its scene: a block per 32
// tiles of the whole array
inline unsigned region_blocks(unsigned tiles) { return std::min(kRegionBlocks, std::max(1u, tiles / 32)); }
// Blocks of an element-wise batched stage over n elements (kBatchVirt lone blocks each)
inline unsigned virt_blocks(size_t n) { return cdiv(cdiv(n, 256), kBatchVirt); }

// Prefix arrays of the step (cap + 1 entries each), in upload order
// (PParticles, PCells, PRows: kBatchVirt lone blocks per batched block; PMove: one)
enum Pre { PAdvect, PAdvFold, PParticles, PMove, PMoveFold, PCells, PSortLarge, PScan, PExtrap, PFill, PUpdU, PUpdV,
           PUpdW, PRows, PTiles, kPre = PTiles + kTileShapes };  // PTiles + k: tiles in tile shape k

struct Layout {
    size_t scenes, args, segs, pre, rows, state, up, total;
    Layout(int cap, size_t argBytes) {
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        scenes = 0;
        args = al((size_t)cap * sizeof(BScene));
        segs = args + al((size_t)cap * argBytes);
        pre = segs + al(2 * (size_t)cap * sizeof(ScanSeg));
        up = pre + al((size_t)kPre * (cap + 1) * sizeof(unsigned));
        rows = up;
        state = rows + al((size_t)cap * sizeof(unsigned));
        total = state + al((size_t)cap * sizeof(DevState));
    }
};

} // namespace

bool batch_step_eligible(const bnn_flip* h) {
    return h->P.solver_kind == BNN_SOLVER_FLIP && !h->gridBoundary && !h->P.correct_position && h->n > 0 &&
           h->P.pcg_mode == BNN_PCG_REFINED && h->moved != nullptr;
}

void batch_step_release(BatchStepWork& w) {
    for(auto& g : w.seg)
        if(g.exec) cudaGraphExecDestroy(g.exec);
    if(w.dev) cudaFree(w.dev);
    if(w.host) cudaFreeHost(w.host);
    for(auto& e : w.ev)
        if(e) cudaEventDestroy(e);
    if(w.s) cudaStreamDestroy(w.s);
    pcg_batch_release(w.pcg);
    w = BatchStepWork();
}

// Runs a segment of launches: directly, or as a CUDA graph captured from them (again when
// the launch shapes `sig` changed since the last capture) and replayed.  A new capture
// with the same launches in the same order (scenes come and go, block counts change) is
// written into the existing executable graph (cudaGraphExecUpdate), which costs far less
// host time than building a new one; only a different sequence of launches is built anew.
template<class F> static int run_segment(StagedGraph& g, const std::vector<uint64_t>& sig, cudaStream_t s,
                                         bool graph, F body) {
    if(!graph) return body(false);
    if(!g.exec || g.sig != sig) {
        const long long l0 = (long long)bnn_launch_count();
        BNN_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int rc = body(true);
        cudaGraph_t cg = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &cg);
        const long long kernels = (long long)bnn_launch_count() - l0;
        bnn_note_launches(-kernels);  // captured, not run
        if(rc != BNN_OK || e != cudaSuccess) {
            if(cg) cudaGraphDestroy(cg);
            if(rc != BNN_OK) return rc;
            BNN_CUDA_CHECK(e);
        }
        bool done = false;
        if(g.exec && kernels == g.kernels) {
            cudaGraphExecUpdateResultInfo info;
            if(cudaGraphExecUpdate(g.exec, cg, &info) == cudaSuccess) {
                done = true;
                ++g.updated;
            } else {
                (void)cudaGetLastError();  // a refused update leaves no error behind
            }
        }
        if(!done) {
            if(g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
            const cudaError_t ei = cudaGraphInstantiate(&g.exec, cg, 0);
            if(ei != cudaSuccess) {
                g.exec = nullptr;
                cudaGraphDestroy(cg);
                BNN_CUDA_CHECK(ei);
            }
            ++g.instantiated;
        }
        cudaGraphDestroy(cg);
        g.kernels = kernels;
        g.sig = sig;
    }
    BNN_CUDA_CHECK(cudaGraphLaunch(g.exec, s));
    bnn_note_launches(g.kernels);
    return BNN_OK;
}

static int batch_reserve(BatchStepWork& w, int ns) {
    if(!w.s) {
        BNN_CUDA_CHECK(cudaStreamCreateWithFlags(&w.s, cudaStreamNonBlocking));
        for(auto& e : w.ev) BNN_CUDA_CHECK(cudaEventCreate(&e));
    }
    if(ns <= w.cap && w.dev) return BNN_OK;
    if(w.dev) cudaFree(w.dev);
    if(w.host) cudaFreeHost(w.host);
    w.dev = w.host = nullptr;
    const int cap = ns < 64 ? 64 : ns + ns / 4;
    const Layout L(cap, p2g_tile_args_bytes());
    BNN_CUDA_CHECK(cudaMalloc(&w.dev, L.total));
    BNN_CUDA_CHECK(cudaMallocHost(&w.host, L.total));
    std::memset(w.host, 0, L.total);
    w.cap = cap;
    return BNN_OK;
}

int batch_substep(BatchStepWork& w, bnn_flip* const* hs, int nsIn, int* rc, bnn_step_stats* st) {
    // scenes whose fused move was sized differently fail alone, as in run_substep
    std::vector<bnn_flip*> sc;
    std::vector<int> at;  // position in hs
    std::vector<float> substep;
    for(int i = 0; i < nsIn; ++i) {
        bnn_flip* h = hs[i];
        rc[i] = BNN_OK;
        std::memset(&st[i], 0, sizeof(bnn_step_stats));
        const float dt = begin_substep(h);
        const bool moved = h->premoved && h->n > 0;
        if(moved && dt != h->premovedDt) {
            drop_premove(h);
            cudaStreamSynchronize(h->s);
            bnn_set_error("sub-step size of the fused move differs from the host's");
            rc[i] = BNN_ERR_DEVICE_CHECK;
            continue;
        }
        // work queued on the scene's own stream finishes before the batch's
        BNN_CUDA_CHECK(cudaStreamSynchronize(h->s));
        sc.push_back(h);
        at.push_back(i);
        substep.push_back(dt);
    }
    const int ns = (int)sc.size();
    if(ns == 0) return BNN_OK;
    int r = batch_reserve(w, ns);
    if(r != BNN_OK) return r;
    const size_t argBytes = p2g_tile_args_bytes();
    const Layout L(w.cap, argBytes);
    char* H = (char*)w.host;
    char* D = (char*)w.dev;
    BScene* hS = (BScene*)(H + L.scenes);
    const BScene* dS = (const BScene*)(D + L.scenes);
    ScanSeg* hSeg = (ScanSeg*)(H + L.segs);
    const ScanSeg* dSeg = (const ScanSeg*)(D + L.segs);
    auto hP = [&](int k) { return (unsigned*)(H + L.pre) + (size_t)k * (w.cap + 1); };
    auto dP = [&](int k) { return (const unsigned*)(D + L.pre) + (size_t)k * (w.cap + 1); };
    auto tot = [&](int k) { return hP(k)[ns]; };
    cudaStream_t s = w.s;

    // ---- the scene table and the prefixes of every stage before the pressure rows
    for(int k = 0; k < kPre; ++k) hP(k)[0] = 0;
    uint64_t cells = 0;
    for(int q = 0; q < ns; ++q) {
        bnn_flip* h = sc[q];
        const float dt = substep[q];
        const bool moved = h->premoved && h->n > 0;
        h->premoved = false;
        BScene& c = hS[q];
        std::memset(&c, 0, sizeof c);
        c.g = h->g;
        c.n = (int)h->n;
        c.advSteps = (int)h->P.advection_steps;
        c.moved = moved ? 1 : 0;
        c.cap = h->cap;
        c.C = h->C;
        c.substep = dt;
        c.sub = dt / (float)h->P.advection_steps;
        c.gdt = h->P.apply_gravity ? 9.81f * dt : 0.f;
        c.ratio = h->P.pic_flip_ratio;
        c.ns.frameTime = h->frameTime + dt;
        c.ns.frameDuration = h->frameDuration;
        c.ns.cfl = h->P.cfl_factor;
        c.ns.minDt = h->P.min_timestep;
        c.ns.maxDt = h->P.max_timestep;
        c.ns.advSteps = (int)h->P.advection_steps;
        c.p6cur = h->p6[h->cur];
        c.p6nxt = h->p6[1 - h->cur];
        c.movedPos = h->moved;
        c.idcur = h->ids[h->cur];
        c.idnxt = h->ids[1 - h->cur];
        c.rec = h->rec;
        c.cellOf = h->cellOf; c.slot = h->slot; c.order = h->order; c.key = h->key;
        c.count = h->count; c.cellStart = h->cellStart;
        c.bboxPart = h->bboxPart;
        for(int d = 0; d < 3; ++d) {
            c.U[d] = h->U[d]; c.B[d] = h->B[d]; c.O[d] = h->O[d]; c.VA[d] = h->VA[d]; c.VB[d] = h->VB[d];
        }
        c.phi = h->phi; c.flag = h->flag; c.aidx = h->aidx;
        c.dst = h->dst;
        p2g_tile_args(H + L.args + (size_t)q * argBytes, h->g, h->dst, h->cellStart, h->rec, h->cap, h->U, h->VA,
                      h->phi);
        if(((uintptr_t)h->count | (uintptr_t)h->cellStart | (uintptr_t)h->flag | (uintptr_t)h->aidx) & 15u) {
            bnn_set_error("batched scan: cell arrays not 16-byte aligned");
            return BNN_ERR_NOT_SUPPORTED;
        }
        hSeg[q] = ScanSeg{h->count, h->cellStart, (uint32_t*)h->scanWs, h->C};
        hSeg[ns + q] = ScanSeg{h->flag, h->aidx, (uint32_t*)h->scanWs, h->C};
        const unsigned pb = virt_blocks((size_t)c.n);
        unsigned tiles[3], ftot = 0;
        size_t fmax = 0;
        for(int d = 0; d < 3; ++d) {
            tiles[d] = region_tiles(h->g, d);
            ftot += tiles[d];
            fmax = std::max(fmax, h->F[d]);
        }
        unsigned add[kPre] = {
            moved ? 0u : pb,                                   // PAdvect
            moved ? 0u : bbox_fold_blocks(c.n),                // PAdvFold
            pb,                                                // PParticles
            cdiv((size_t)c.n, 256),                            // PMove
            bbox_fold_blocks(c.n),                             // PMoveFold
            virt_blocks(h->C),                                 // PCells
            c.n > 16 ? std::min(296u, std::max(2u, cdiv((size_t)c.n, 8192))) : 0u,  // PSortLarge
            cdiv(h->C, kScanSegTile),                          // PScan
            region_blocks(ftot),                               // PExtrap
            std::min(kRegionBlocks, cdiv(fmax, 2048)),         // PFill
            region_blocks(tiles[0]), region_blocks(tiles[1]), region_blocks(tiles[2]),  // PUpd*
            0u};                                               // PRows (after the numbering)
        for(int k = 0; k < kTileShapes; ++k) add[PTiles + k] = p2g_sdf_tiles(h->g, k);
        for(int k = 0; k < kPre; ++k) hP(k)[q + 1] = hP(k)[q] + add[k];
        cells += h->C;
    }
    BNN_CUDA_CHECK(cudaMemcpyAsync(D, H, L.up, cudaMemcpyHostToDevice, s));

    // ---- segment 1: move, counting sort, P2G + fluid SDF, extrapolation, numbering
    const int shape = p2g_batch_shape(ns, cells);
    const bool capture = w.graphs && shape >= 0;  // the tuner synchronises: not inside a capture
    unsigned* dRows = (unsigned*)(D + L.rows);
    const unsigned* hRows = (const unsigned*)(H + L.rows);
    cudaEventRecord(w.ev[0], s);
    auto seg1 = [&](bool capturing) -> int {
        auto mark = [&](int k) { capturing ? cudaEventRecordWithFlags(w.ev[k], s, cudaEventRecordExternal)
                                           : cudaEventRecord(w.ev[k], s); };
        launch_batch_stage(BatchStage::StepReset, dS, nullptr, ns, 0, s);
        launch_batch_stage(BatchStage::Advect, dS, dP(PAdvect), ns, tot(PAdvect), s);
        launch_batch_stage(BatchStage::BboxFinal, dS, dP(PAdvFold), ns, tot(PAdvFold), s);
        mark(1);
        BNN_CUDA_CHECK(batched_exclusive_scan_u32(dSeg, dP(PScan), ns, tot(PScan), s));
        launch_batch_stage(BatchStage::ScatterIndex, dS, dP(PParticles), ns, tot(PParticles), s);
        launch_batch_stage(BatchStage::SortBuckets, dS, dP(PCells), ns, tot(PCells), s);
        launch_batch_stage(BatchStage::SortLarge, dS, dP(PSortLarge), ns, tot(PSortLarge), s);
        launch_batch_stage(BatchStage::Gather, dS, dP(PParticles), ns, tot(PParticles), s);
        mark(2);
        {
            const unsigned* P[kTileShapes];
            unsigned tiles[kTileShapes];
            for(int k = 0; k < kTileShapes; ++k) {
                P[k] = dP(PTiles + k);
                tiles[k] = tot(PTiles + k);
            }
            launch_p2g_sdf_batch(D + L.args, P, tiles, ns, cells, s);
        }
        mark(3);
        // extrapolate, backup, gravity (FLIP_Solver.cpp:44-47)
        for(int layer = 0; layer < 4; ++layer) {
            if(layer == 3) launch_batch_stage(BatchStage::FillBackup, dS, dP(PFill), ns, tot(PFill), s);
            launch_batch_stage(BatchStage::Extrapolate, dS, dP(PExtrap), ns, tot(PExtrap), s, 1, layer);
        }
        mark(4);
        mark(5);
        // the pressure system's numbering, and its row count per scene to the host
        launch_batch_stage(BatchStage::ActiveFlags, dS, dP(PCells), ns, tot(PCells), s);
        BNN_CUDA_CHECK(batched_exclusive_scan_u32(dSeg + ns, dP(PScan), ns, tot(PScan), s));
        launch_batch_gather_rows(dS, ns, dRows, s);
        BNN_CUDA_CHECK(cudaMemcpyAsync(H + L.rows, dRows, (size_t)ns * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        return BNN_OK;
    };
    {
        const std::vector<uint64_t> sig = {(uint64_t)(uintptr_t)w.dev, (uint64_t)w.cap, (uint64_t)ns, (uint64_t)shape,
                                           tot(PAdvect), tot(PAdvFold), tot(PScan), tot(PParticles), tot(PCells),
                                           tot(PSortLarge), tot(PTiles + (shape < 0 ? 0 : shape)), tot(PExtrap),
                                           tot(PFill)};
        r = run_segment(w.seg[0], sig, s, capture, seg1);
        if(r != BNN_OK) return r;
    }
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    // rows of every scene, then the table again (row arrays may have moved)
    std::vector<BatchSolveItem> items(ns);
    for(int q = 0; q < ns; ++q) {
        bnn_flip* h = sc[q];
        const uint32_t nrows = hRows[q];
        r = reserve_rows(h, nrows);
        if(r != BNN_OK) return r;
        h->nRows = nrows;
        BScene& c = hS[q];
        c.nrows = (int)nrows;
        c.rowCell = h->rowCell; c.rhs = h->rhs; c.diag = h->diag; c.invd = h->invd; c.pressure = h->pressure;
        c.nbr = h->nbr;
        hP(PRows)[q + 1] = hP(PRows)[q] + virt_blocks(nrows);
        BatchSolveItem& it = items[q];
        it.w = &h->pcg;
        it.n = (int)nrows;
        it.rhs = h->rhs; it.diag = h->diag; it.invd = h->invd; it.nbr = h->nbr;
        it.dt = substep[q];
        it.innerTol = h->P.refine_inner_tolerance;
        it.outerTol = h->P.refine_tolerance;
        it.maxIter = h->P.max_cg_iteration;
        it.pressure = h->pressure;
        it.dst = h->dst;
    }
    BNN_CUDA_CHECK(cudaMemcpyAsync(D, H, L.up, cudaMemcpyHostToDevice, s));
    launch_batch_stage(BatchStage::ActiveRows, dS, dP(PCells), ns, tot(PCells), s);
    launch_batch_stage(BatchStage::BuildRows, dS, dP(PRows), ns, tot(PRows), s);
    cudaEventRecord(w.ev[6], s);
    // ---- pressure: the refined solves of all scenes
    r = pcg_solve_batch_refined(w.pcg, items.data(), ns, s);
    if(r != BNN_OK) return r;
    cudaEventRecord(w.ev[7], s);
    // ---- segment 2: projection, extrapolation of the projected faces, CFL maximum, the
    // grid-to-particle transfer + the next sub-step's move, the scenes' state to the host
    DevState* dState = (DevState*)(D + L.state);
    const DevState* hState = (const DevState*)(H + L.state);
    auto seg2 = [&](bool capturing) -> int {
        auto mark = [&](int k) { capturing ? cudaEventRecordWithFlags(w.ev[k], s, cudaEventRecordExternal)
                                           : cudaEventRecord(w.ev[k], s); };
        launch_batch_stage(BatchStage::FillUpdate, dS, dP(PFill), ns, tot(PFill), s);
        launch_batch_stage(BatchStage::UpdateU, dS, dP(PUpdU), ns, tot(PUpdU), s);
        launch_batch_stage(BatchStage::UpdateV, dS, dP(PUpdV), ns, tot(PUpdV), s);
        launch_batch_stage(BatchStage::UpdateW, dS, dP(PUpdW), ns, tot(PUpdW), s);
        for(int layer = 0; layer < 4; ++layer)
            launch_batch_stage(BatchStage::Extrapolate, dS, dP(PExtrap), ns, tot(PExtrap), s, 2, layer);
        mark(8);
        launch_batch_stage(BatchStage::BboxReset, dS, nullptr, ns, 0, s);
        launch_batch_stage(BatchStage::G2PMove, dS, dP(PMove), ns, tot(PMove), s);
        launch_batch_stage(BatchStage::BboxFinal, dS, dP(PMoveFold), ns, tot(PMoveFold), s);
        mark(9);
        launch_batch_gather_state(dS, ns, dState, s);
        BNN_CUDA_CHECK(cudaMemcpyAsync(H + L.state, dState, (size_t)ns * sizeof(DevState), cudaMemcpyDeviceToHost, s));
        return BNN_OK;
    };
    {
        const std::vector<uint64_t> sig = {(uint64_t)(uintptr_t)w.dev, (uint64_t)w.cap, (uint64_t)ns, tot(PFill),
                                           tot(PUpdU), tot(PUpdV), tot(PUpdW), tot(PExtrap), tot(PMove),
                                           tot(PMoveFold)};
        r = run_segment(w.seg[1], sig, s, w.graphs, seg2);
        if(r != BNN_OK) return r;
    }
    BNN_CUDA_CHECK(cudaGetLastError());
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));

    float stage[10] = {};
    {
        const int map[10][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {7, 8}, {8, 9}, {0, 9}};
        for(int k = 0; k < 10; ++k) cudaEventElapsedTime(&stage[k], w.ev[map[k][0]], w.ev[map[k][1]]);
    }
    // ---- the host side of the step's end, scene by scene (run_substep's)
    for(int q = 0; q < ns; ++q) {
        bnn_flip* h = sc[q];
        const float dt = substep[q];
        *h->hst = hState[q];
        h->cur = 1 - h->cur;
        for(int d = 0; d < 3; ++d) {
            std::swap(h->U[d], h->B[d]);
            std::swap(h->VA[d], h->VB[d]);
        }
        h->maxvelBits = h->hst->maxvel_bits;
        h->frameTime += dt;
        ++h->substepIndex;
        h->premoved = true;
        h->premovedDt = h->hst->next_dt;
        const PcgOutcome& po = items[q].out;
        bnn_step_stats& o = st[at[q]];
        o.dt = dt;
        o.frame_time = h->frameTime;
        o.frame_finished = h->frameTime >= h->frameDuration ? 1u : 0u;
        o.pcg_iterations = po.iterations;
        o.pcg_residual = po.residual;
        o.pcg_success = po.success;
        o.n_active = h->nRows;
        o.outer_iterations = po.outer;
        o.pcg_kernel_ms = po.kernelMs;
        o.zero_phi_cells = h->hst->zero_phi;
        o.device_flags = h->hst->flags;
        for(int k = 0; k < 10; ++k) o.stage_ms[k] = stage[k];
        int& e = rc[at[q]];
        if(h->hst->flags & BNN_FLAG_OUT_OF_GRID) e = BNN_ERR_DEVICE_CHECK;
        else if(!po.success) e = BNN_ERR_PCG_NOT_CONVERGED;
    }
    return BNN_OK;
}
