// bnn_flip_run: run a scene file through FLIP_GPU_Solver the way the reference's
// Simulator does (ParticleSolverFactory::createSolverFromJSon, loadScene, doFrameSimulation
// per frame, finalizeSimulation; Simulator.cpp:38-69), print one JSON line per frame and
// write the final particles.
//
//   bnn_flip_run scene.json [--frames N] [--out particles.f32]
//   bnn_flip_run scene.json --sample-only particles.f32   (generated particles, no GPU)
//
// The output file holds uint32 n, then n*3 float32 positions and n*3 float32 velocities.
#include "FLIP_GPU_Solver.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

int main(int argc, char** argv) {
    if(argc < 2) {
        std::fprintf(stderr, "usage: %s scene.json [--frames N] [--out file]\n", argv[0]);
        return 2;
    }
    std::string scene = argv[1], out, sampleOnly;
    long frames = -1;
    for(int a = 2; a + 1 < argc; a += 2) {
        if(!std::strcmp(argv[a], "--frames")) frames = std::atol(argv[a + 1]);
        else if(!std::strcmp(argv[a], "--out")) out = argv[a + 1];
        else if(!std::strcmp(argv[a], "--sample-only")) sampleOnly = argv[a + 1];
    }
    auto write_particles = [](const std::string& path, bnnhost::ParticleData& D) {
        std::FILE* fo = std::fopen(path.c_str(), "wb");
        if(!fo) return false;
        const uint32_t n = D.getNParticles();
        std::fwrite(&n, sizeof(n), 1, fo);
        std::fwrite(D.positions.data(), sizeof(float), 3 * (size_t)n, fo);
        std::fwrite(D.velocities.data(), sizeof(float), 3 * (size_t)n, fo);
        std::fclose(fo);
        return true;
    };
    auto solver = bnnhost::ParticleSolverFactory::createSolverFromJSon(scene);
    if(!solver) {
        std::fprintf(stderr, "the solver named in '%s' is not supported\n", scene.c_str());
        return 1;
    }
    if(!sampleOnly.empty()) {
        solver->loadScene(scene, false);
        return write_particles(sampleOnly, solver->generalParticleData()) ? 0 : 1;
    }
    solver->loadScene(scene);
    auto& G = solver->globalParams();
    if(frames > 0) G.finalFrame = G.startFrame + (unsigned)frames - 1;
    std::printf("{\"solver\": \"%s\", \"particles\": %u, \"resumed_after_frame\": %u}\n",
                solver->getSolverName().c_str(), solver->generalParticleData().getNParticles(), G.finishedFrame);
    // a scene that resumes from a memory state continues after the state's frame
    const unsigned first = G.startFrame > G.finishedFrame + 1 ? G.startFrame : G.finishedFrame + 1;
    for(unsigned f = first; f <= G.finalFrame; ++f) {
        const auto t0 = std::chrono::steady_clock::now();
        solver->doFrameSimulation(f);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        const auto& L = solver->frameLogs().back();
        std::printf("{\"frame\": %u, \"substeps\": %u, \"pcg_iterations\": %u, \"residual\": %.6g, "
                    "\"gpu_ms\": %.3f, \"wall_ms\": %.3f}\n",
                    f, L.substeps, L.pcgIterations, L.lastResidual, L.gpuMs, ms);
        std::fflush(stdout);
    }
    if(!out.empty() && !write_particles(out, solver->generalParticleData())) {
        std::fprintf(stderr, "cannot write %s\n", out.c_str());
        return 1;
    }
    solver->finalizeSimulation();
    return 0;
}
