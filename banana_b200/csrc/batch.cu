// Scene batches: many independent FLIP scenes stepped together on one GPU.
//
// Every scene is a full solver handle (its own grids, particles, pressure system and CUDA
// stream), so each scene computes exactly what a lone bnn_flip_step computes.  A step of
// the batch advances every live scene by one sub-step:
// * the scenes the staged step takes (batch_step.cu) advance together on the batch's own
//   stream, one kernel launch per stage of the sub-step over all of them;
// * the others (and all of them in BNN_BATCH_PER_SCENE mode) are stepped by a pool of host
//   worker threads (longest first, to the least loaded worker), each scene on its own
//   stream, so the kernels of many small scenes run side by side.
// Both run at the same time; the cooperative PCG launches of the two share the GPU through
// pcg.cu's occupancy accounting.  Scenes are admitted against a device-memory budget with
// bnn_scene_bytes_estimate.
//
// The reference runs one scene per ParticleSolver object (ParticleSolver.h:39-105); a
// batch is what a server holding many such objects does, with the objects on one GPU.
#include "batch_step.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct Scene {
    uint32_t id = 0;
    bnn_flip* h = nullptr;
    uint64_t estimate = 0;
    uint32_t n = 0;
    uint64_t steps = 0;
    int status = BNN_OK;
    double ms = 0.0;  // host wall time of its last step
    bnn_step_stats last{};
};

} // namespace

struct bnn_batch {
    int device = 0;
    uint32_t mode = BNN_BATCH_STAGED;
    BatchStepWork staged;
    uint64_t budget = 0;
    uint64_t admitted = 0;
    uint32_t nextId = 1;
    std::vector<std::unique_ptr<Scene>> scenes;
    // worker pool
    int nworkers = 1;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    uint64_t gen = 0;
    int pending = 0;
    bool quit = false;
    std::vector<std::vector<Scene*>> work;

    void worker(int w) {
        cudaSetDevice(device);
        uint64_t seen = 0;
        for(;;) {
            std::vector<Scene*> mine;
            {
                std::unique_lock<std::mutex> lk(mu);
                cvWork.wait(lk, [&] { return quit || gen != seen; });
                if(quit) return;
                seen = gen;
                mine = work[w];
            }
            for(Scene* sc : mine) {
                const auto t0 = std::chrono::steady_clock::now();
                sc->status = bnn_flip_step(sc->h, &sc->last);
                sc->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                if(sc->status == BNN_OK) ++sc->steps;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                if(--pending == 0) cvDone.notify_all();
            }
        }
    }
};

static Scene* find_scene(bnn_batch* b, uint32_t id) {
    for(auto& s : b->scenes)
        if(s->id == id) return s.get();
    return nullptr;
}

extern "C" int bnn_batch_create(const bnn_batch_params* params, bnn_batch** out) {
    if(!out) return BNN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const uint32_t mode = params ? params->step_mode : BNN_BATCH_STAGED;
    if(((mode & 0xffu) != BNN_BATCH_STAGED && (mode & 0xffu) != BNN_BATCH_PER_SCENE) ||
       (mode & ~(0xffu | BNN_BATCH_NO_GRAPHS))) {
        bnn_set_error("bnn_batch_create: unknown step_mode");
        return BNN_ERR_INVALID_ARGUMENT;
    }
    int device = 0;
    BNN_CUDA_CHECK(cudaGetDevice(&device));
    auto* b = new bnn_batch();
    b->device = device;
    b->budget = params ? params->hbm_budget_bytes : 0;
    b->mode = mode & 0xffu;
    b->staged.graphs = (mode & BNN_BATCH_NO_GRAPHS) == 0;
    int nw = params && params->worker_threads ? (int)params->worker_threads : 0;
    if(nw <= 0) {
        const unsigned hc = std::thread::hardware_concurrency();
        nw = (int)std::min(16u, hc ? hc : 4u);
    }
    b->nworkers = nw;
    b->work.resize(nw);
    for(int w = 0; w < nw; ++w) b->threads.emplace_back([b, w] { b->worker(w); });
    *out = b;
    return BNN_OK;
}

extern "C" int bnn_batch_destroy(bnn_batch* b) {
    if(!b) return BNN_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        b->quit = true;
    }
    b->cvWork.notify_all();
    for(auto& t : b->threads) t.join();
    batch_step_release(b->staged);
    for(auto& s : b->scenes) bnn_flip_destroy(s->h);
    delete b;
    return BNN_OK;
}

extern "C" int bnn_batch_add_scene(bnn_batch* b, const bnn_params* params, const float* pos, const float* vel,
                                   uint32_t n, uint32_t* id_out) {
    if(!b || !params || !id_out || (n && (!pos || !vel))) return BNN_ERR_INVALID_ARGUMENT;
    uint64_t est = 0;
    int rc = bnn_scene_bytes_estimate(params, n, &est);
    if(rc != BNN_OK) return rc;
    if(b->budget && b->admitted + est > b->budget) {
        bnn_set_error("bnn_batch_add_scene: the scene does not fit the device-memory budget");
        return BNN_ERR_CAPACITY;
    }
    BNN_CUDA_CHECK(cudaSetDevice(b->device));
    bnn_flip* h = nullptr;
    rc = bnn_flip_create(params, &h);
    if(rc != BNN_OK) return rc;
    rc = bnn_flip_set_particles(h, pos, vel, n);
    if(rc != BNN_OK) { bnn_flip_destroy(h); return rc; }
    auto s = std::make_unique<Scene>();
    s->id = b->nextId++;
    s->h = h;
    s->estimate = est;
    s->n = n;
    b->admitted += est;
    *id_out = s->id;
    b->scenes.push_back(std::move(s));
    return BNN_OK;
}

extern "C" int bnn_batch_remove_scene(bnn_batch* b, uint32_t id) {
    if(!b) return BNN_ERR_INVALID_ARGUMENT;
    for(size_t i = 0; i < b->scenes.size(); ++i) {
        if(b->scenes[i]->id != id) continue;
        bnn_flip_destroy(b->scenes[i]->h);
        b->admitted -= b->scenes[i]->estimate;
        b->scenes.erase(b->scenes.begin() + (long)i);
        return BNN_OK;
    }
    return BNN_ERR_INVALID_ARGUMENT;
}

extern "C" int bnn_batch_step(bnn_batch* b, bnn_batch_stats* stats) {
    if(!b) return BNN_ERR_INVALID_ARGUMENT;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<Scene*> staged, rest;
    for(auto& s : b->scenes)
        (b->mode == BNN_BATCH_STAGED && batch_step_eligible(s->h) ? staged : rest).push_back(s.get());
    {
        std::unique_lock<std::mutex> lk(b->mu);
        // longest processing time first: biggest scene to the least loaded worker
        std::stable_sort(rest.begin(), rest.end(), [](const Scene* x, const Scene* y) { return x->estimate > y->estimate; });
        std::vector<uint64_t> load(b->nworkers, 0);
        for(auto& w : b->work) w.clear();
        for(Scene* s : rest) {
            const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            b->work[w].push_back(s);
            load[w] += s->estimate;
        }
        b->pending = b->nworkers;
        ++b->gen;
    }
    b->cvWork.notify_all();
    int batchRc = BNN_OK;
    unsigned long long inst0 = 0, upd0 = 0;
    for(const auto& g : b->staged.seg) { inst0 += g.instantiated; upd0 += g.updated; }
    if(!staged.empty()) {
        // the staged scenes on this thread, meanwhile
        const int ns = (int)staged.size();
        std::vector<bnn_flip*> hs(ns);
        std::vector<int> rcs(ns);
        std::vector<bnn_step_stats> sts(ns);
        for(int i = 0; i < ns; ++i) hs[i] = staged[i]->h;
        const auto t1 = std::chrono::steady_clock::now();
        batchRc = batch_substep(b->staged, hs.data(), ns, rcs.data(), sts.data());
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
        for(int i = 0; i < ns; ++i) {
            Scene* sc = staged[i];
            sc->status = batchRc != BNN_OK ? batchRc : rcs[i];
            sc->last = sts[i];
            sc->ms = ms;
            if(sc->status == BNN_OK) ++sc->steps;
        }
    }
    {
        std::unique_lock<std::mutex> lk(b->mu);
        b->cvDone.wait(lk, [&] { return b->pending == 0; });
    }
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    int rc = batchRc;
    bnn_batch_stats st{};
    st.wall_ms = wall;
    st.staged_scenes = (uint32_t)staged.size();
    {
        unsigned long long inst1 = 0, upd1 = 0;
        for(const auto& g : b->staged.seg) { inst1 += g.instantiated; upd1 += g.updated; }
        st.graph_instantiations = (uint16_t)(inst1 - inst0);
        st.graph_updates = (uint16_t)(upd1 - upd0);
    }
    for(auto& s : b->scenes) {
        ++st.scenes;
        if(s->status != BNN_OK) {
            ++st.failed;
            if(rc == BNN_OK) rc = s->status;
            continue;
        }
        st.particle_steps += s->n;
        st.pcg_iterations += s->last.pcg_iterations;
        st.max_scene_ms = std::max(st.max_scene_ms, s->ms);
    }
    if(stats) *stats = st;
    return rc;
}

extern "C" int bnn_batch_scene_info(bnn_batch* b, uint32_t id, uint32_t* n, uint64_t* steps, bnn_step_stats* last) {
    if(!b) return BNN_ERR_INVALID_ARGUMENT;
    Scene* s = find_scene(b, id);
    if(!s) return BNN_ERR_INVALID_ARGUMENT;
    if(n) *n = s->n;
    if(steps) *steps = s->steps;
    if(last) *last = s->last;
    return s->status;
}

extern "C" int bnn_batch_get_scene(bnn_batch* b, uint32_t id, float* pos, float* vel) {
    if(!b) return BNN_ERR_INVALID_ARGUMENT;
    Scene* s = find_scene(b, id);
    if(!s) return BNN_ERR_INVALID_ARGUMENT;
    return bnn_flip_get_particles(s->h, pos, vel);
}

extern "C" int bnn_batch_memory(bnn_batch* b, uint64_t* admitted, uint64_t* held) {
    if(!b) return BNN_ERR_INVALID_ARGUMENT;
    if(admitted) *admitted = b->admitted;
    if(held) {
        uint64_t t = 0;
        for(auto& s : b->scenes) {
            uint64_t x = 0;
            bnn_flip_device_bytes(s->h, &x);
            t += x;
        }
        *held = t;
    }
    return BNN_OK;
}
