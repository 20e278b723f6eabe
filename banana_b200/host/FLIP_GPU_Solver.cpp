// FLIP_GPU_Solver: ParticleSolver-shaped host class over the banana_b200 C ABI.
#include "FLIP_GPU_Solver.h"

#include "bnn_io.h"
#include "json_lite.h"

#include <future>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace bnnhost {

// ---------------------------------------------------------------------------------
// seeded sampling (must match banana_b200/scenes.py: dam_break / uniform01 / splitmix64)
// ---------------------------------------------------------------------------------
static inline uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double uniform01(uint64_t seed, uint64_t stream, uint64_t counter) {
    const uint64_t key = splitmix64(seed * 0x9E3779B97F4A7C15ull + stream * 0xD1B54A32D192ED03ull);
    const uint64_t bits = splitmix64(counter ^ key);
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

void sample_box(const float domainMin[3], double cellSize, const double bmin[3], const double bmax[3], unsigned ppc,
                uint64_t seed, std::vector<float>& pos, std::vector<float>& vel) {
    int64_t c0[3], nc[3];
    for(int a = 0; a < 3; ++a) {
        const double lo = (bmin[a] - (double)domainMin[a]) / cellSize, hi = (bmax[a] - (double)domainMin[a]) / cellSize;
        c0[a] = (int64_t)std::ceil(lo - 1e-9);
        const int64_t c1 = (int64_t)std::floor(hi + 1e-9);  // one past the last cell
        nc[a] = c1 > c0[a] ? c1 - c0[a] : 0;
    }
    const int64_t ncell = nc[0] * nc[1] * nc[2];
    if(ncell <= 0) return;
    const size_t base = pos.size();
    pos.resize(base + (size_t)ncell * ppc * 3);
    vel.resize(base + (size_t)ncell * ppc * 3, 0.f);
    for(int64_t cell = 0; cell < ncell; ++cell) {
        const int64_t ci[3] = {cell % nc[0], (cell / nc[0]) % nc[1], cell / (nc[0] * nc[1])};
        for(unsigned k = 0; k < ppc; ++k) {
            const uint64_t lin = (uint64_t)(cell * (int64_t)ppc + k);
            for(int a = 0; a < 3; ++a) {
                const double cc = (double)(c0[a] + ci[a]);
                const double u = uniform01(seed, (uint64_t)a, lin);
                float p = (float)((double)domainMin[a] + (cc + u) * cellSize);
                // rounding to float may land a sample on the next cell's face: keep it inside
                const float hi = (float)((double)domainMin[a] + (cc + 1.0) * cellSize);
                if(p >= hi) p = std::nextafter(hi, 0.0f);
                pos[base + ((size_t)lin) * 3 + (size_t)a] = p;
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// factory
// ---------------------------------------------------------------------------------
std::map<std::string, ParticleSolverFactory::CreateMethod>& ParticleSolverFactory::methods() {
    static std::map<std::string, CreateMethod> m;
    return m;
}

bool ParticleSolverFactory::registerSolver(const std::string& name, CreateMethod create) {
    methods()[name] = std::move(create);
    return true;
}

std::shared_ptr<FLIP_GPU_Solver> ParticleSolverFactory::createSolver(const std::string& name) {
    auto it = methods().find(name);
    return it == methods().end() ? nullptr : it->second();
}

static std::string read_file(const std::string& path) {
    std::ifstream f(path);
    if(!f) throw std::runtime_error("cannot open scene file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

std::shared_ptr<FLIP_GPU_Solver> ParticleSolverFactory::createSolverFromJSon(const std::string& sceneFile) {
    const Json j = JsonParser(read_file(sceneFile)).parse();
    std::string name;
    if(!read_string(j["GlobalParameters"], "Solver", name)) return nullptr;
    return createSolver(name);
}

// static registration, as RegisteredInSolverFactory does (ParticleSolverFactory.h:51-60)
static const bool s_registered = ParticleSolverFactory::registerSolver(FLIP_GPU_Solver::solverName(), [] {
    return std::make_shared<FLIP_GPU_Solver>();
}) && ParticleSolverFactory::registerSolver(APIC_GPU_Solver::solverName(), [] {
    return std::static_pointer_cast<FLIP_GPU_Solver>(std::make_shared<APIC_GPU_Solver>());
}) && ParticleSolverFactory::registerSolver(AFLIP_GPU_Solver::solverName(), [] {
    return std::static_pointer_cast<FLIP_GPU_Solver>(std::make_shared<AFLIP_GPU_Solver>());
}) && ParticleSolverFactory::registerSolver(PIC_GPU_Solver::solverName(), [] {
    return std::static_pointer_cast<FLIP_GPU_Solver>(std::make_shared<PIC_GPU_Solver>());
});

// ---------------------------------------------------------------------------------
// solver
// ---------------------------------------------------------------------------------
FLIP_GPU_Solver::~FLIP_GPU_Solver() {
    if(m_Gpu) bnn_flip_destroy(m_Gpu);
}

void FLIP_GPU_Solver::check(int status, const char* what) {
    if(status == BNN_OK) return;
    std::fprintf(stderr, "%s: %s failed with status %d (%s)\n", getSolverName().c_str(), what, status,
                 bnn_last_error());
    if(status == BNN_ERR_PCG_NOT_CONVERGED) {
        // PIC_Solver::solveSystem logs the failure and exits only when asked to
        if(m_SolverParams.bExitIfPressureProjectionFailed) std::exit(EXIT_FAILURE);
        return;
    }
    std::exit(EXIT_FAILURE);  // __BNN_REQUIRE
}

void FLIP_GPU_Solver::loadScene(const std::string& sceneFile, bool allocate) {
    loadSceneFromString(read_file(sceneFile), allocate);
}

// ParticleSolver::loadScene (ParticleSolver.cpp:36-130): global and simulation parameters,
// domain box, particle generators, then the solver memory
void FLIP_GPU_Solver::loadSceneFromString(const std::string& sceneJson, bool allocate) {
    const Json j = JsonParser(sceneJson).parse();
    if(!j.has("GlobalParameters") || !j.has("SimulationParameters")) {
        std::fprintf(stderr, "scene needs GlobalParameters and SimulationParameters\n");
        std::exit(EXIT_FAILURE);
    }
    const Json& g = j["GlobalParameters"];
    auto& G = m_GlobalParams;
    read_string(g, "Solver", G.solverName);
    read_value(g, "FrameDuration", G.frameDuration);
    read_value(g, "StartFrame", G.startFrame);
    read_value(g, "FinalFrame", G.finalFrame);
    read_bool(g, "ApplyGravity", G.bApplyGravity);
    read_bool(g, "SaveFrameData", G.bSaveFrameData);
    read_bool(g, "SaveMemoryState", G.bSaveMemoryState);
    read_bool(g, "LoadMemoryState", G.bLoadMemoryState);
    read_value(g, "FramePerState", G.framePerState);
    if(G.framePerState == 0) G.framePerState = 1;
    read_string(g, "DataPath", G.dataPath);
    read_string(g, "FrameDataFolder", G.frameDataFolder);
    read_string(g, "MemoryStateDataFolder", G.memoryStateDataFolder);
    G.SaveDataList.clear();
    const Json& opt = g["OptionalSavingData"];
    for(size_t q = 0; q < opt.size(); ++q)
        if(opt[q].kind == Json::String) G.SaveDataList.push_back(opt[q].str);

    const Json& s = j["SimulationParameters"];
    auto& P = m_SolverParams;
    read_value(s, "MinTimestep", P.minTimestep);
    read_value(s, "MaxTimestep", P.maxTimestep);
    read_value(s, "CFLFactor", P.CFLFactor);
    read_value(s, "CellSize", P.cellSize);
    m_CellSizeScene = (double)P.cellSize;
    read_number(s, "CellSize", m_CellSizeScene);
    read_value(s, "RatioCellSizePRadius", P.ratioCellSizePRadius);
    read_value(s, "NExpandCells", P.nExpandCells);
    read_value(s, "MaxNParticles", P.maxNParticles);
    read_value(s, "AdvectionSteps", P.advectionSteps);
    read_bool(s, "CorrectPosition", P.bCorrectPosition);
    read_value(s, "RepulsiveForceStiffness", P.repulsiveForceStiffness);
    read_value(s, "CGRelativeTolerance", P.CGRelativeTolerance);
    read_value(s, "MaxCGIteration", P.maxCGIteration);
    read_value(s, "PIC_FLIP_ratio", P.PIC_FLIP_ratio);
    read_bool(s, "ExitIfPressureProjectionFailed", P.bExitIfPressureProjectionFailed);
    std::string mode;
    if(read_string(s, "GPU_PCGPrecision", mode))
        P.pcgMode = mode == "fp64" ? BNN_PCG_FP64 : (mode == "refined" ? BNN_PCG_REFINED : BNN_PCG_FP32);
    read_value(s, "GPU_RefineTolerance", P.refineTolerance);
    read_value(s, "GPU_RefineInnerTolerance", P.refineInnerTolerance);
    if(s.has("SimulationDomainBox")) {
        read_vec3(s["SimulationDomainBox"], "BoxMin", P.domainBMin);
        read_vec3(s["SimulationDomainBox"], "BoxMax", P.domainBMax);
    }
    // SimulationParameters::makeReady (ParticleSolverData.cpp:229-272)
    for(int d = 0; d < 3; ++d) {
        P.movingBMin[d] = P.domainBMin[d];
        P.movingBMax[d] = P.domainBMax[d];
    }
    P.particleRadius = P.cellSize / P.ratioCellSizePRadius;

    std::string err;
    m_Boundaries = parse_boundary_objects(j, err);
    if(!err.empty()) {
        std::fprintf(stderr, "%s\n", err.c_str());
        std::exit(EXIT_FAILURE);
    }
    generateParticles(j);
    if(!allocate) return;
    allocateSolverMemory();
    if(G.bLoadMemoryState) {
        const int frame = loadMemoryState();
        if(frame > 0) G.finishedFrame = (unsigned)frame;
    }
}

// ParticleSolver::generateParticles (ParticleSolver.cpp:302-310) for box generators
void FLIP_GPU_Solver::generateParticles(const Json& scene) {
    auto& D = m_ParticleData;
    D.positions.clear();
    D.velocities.clear();
    D.objectIndex.clear();
    D.nObjects = 0;
    const Json& gens = scene["ParticleGenerators"];
    for(size_t q = 0; q < gens.size(); ++q) {
        const Json& o = gens[q];
        std::string type = "Box";
        read_string(o, "GeometryType", type);
        if(type != "Box") {
            std::fprintf(stderr, "%s: particle generator geometry '%s' is not supported (Box only)\n",
                         getSolverName().c_str(), type.c_str());
            std::exit(EXIT_FAILURE);
        }
        double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
        read_vec3(o, "BoxMin", bmin);
        read_vec3(o, "BoxMax", bmax);
        unsigned ppc = 8;
        read_value(o, "ParticlesPerCell", ppc);
        uint64_t seed = 42;
        read_value(o, "Seed", seed);
        const size_t before = D.positions.size() / 3;
        sample_box(m_SolverParams.domainBMin, m_CellSizeScene, bmin, bmax, ppc, seed, D.positions, D.velocities);
        D.objectIndex.resize(D.positions.size() / 3, (int16_t)D.nObjects);
        (void)before;
        ++D.nObjects;
    }
}

void FLIP_GPU_Solver::setParticles(const std::vector<float>& pos, const std::vector<float>& vel) {
    m_ParticleData.positions = pos;
    m_ParticleData.velocities = vel;
    m_ParticleData.objectIndex.assign(pos.size() / 3, 0);
    if(m_Gpu) check(bnn_flip_set_particles(m_Gpu, pos.data(), vel.data(), (uint32_t)(pos.size() / 3)),
                    "bnn_flip_set_particles");
}

// FLIP_Solver::allocateSolverMemory + PIC_Data::makeReady: the device solver
void FLIP_GPU_Solver::allocateSolverMemory() {
    const auto& P = m_SolverParams;
    bnn_params p;
    std::memset(&p, 0, sizeof(p));
    for(int d = 0; d < 3; ++d) {
        p.box_min[d] = P.domainBMin[d];
        p.box_max[d] = P.domainBMax[d];
    }
    p.cell_size = P.cellSize;
    p.n_expand_cells = P.nExpandCells;
    p.cfl_factor = P.CFLFactor;
    p.min_timestep = P.minTimestep;
    p.max_timestep = P.maxTimestep;
    p.frame_duration = m_GlobalParams.frameDuration;
    p.pic_flip_ratio = P.PIC_FLIP_ratio;
    p.cg_relative_tolerance = P.CGRelativeTolerance;
    p.max_cg_iteration = P.maxCGIteration;
    p.advection_steps = P.advectionSteps;
    p.solver_kind = m_SolverKind;
    p.pcg_mode = P.pcgMode;
    p.preconditioner = BNN_PRECOND_JACOBI;
    p.refine_tolerance = P.refineTolerance;
    p.refine_inner_tolerance = P.refineInnerTolerance;
    p.apply_gravity = m_GlobalParams.bApplyGravity ? 1 : 0;
    p.max_particles = P.maxNParticles;
    p.correct_position = P.bCorrectPosition ? 1 : 0;
    p.repulsive_force_stiffness = P.repulsiveForceStiffness;
    p.ratio_cell_size_p_radius = P.ratioCellSizePRadius;
    if(m_Gpu) bnn_flip_destroy(m_Gpu);
    m_Gpu = nullptr;
    check(bnn_flip_create(&p, &m_Gpu), "bnn_flip_create");
    const auto& D = m_ParticleData;
    check(bnn_flip_set_particles(m_Gpu, D.positions.data(), D.velocities.data(), D.getNParticles()),
          "bnn_flip_set_particles");
    // the objects as built (their static transformation); the boundary SDF stays 0 until
    // the scene first moves, as in the reference
    if(!m_Boundaries.empty()) sendBoundaries(false);
}

void FLIP_GPU_Solver::sendBoundaries(bool updateGrid) {
    std::vector<bnn_boundary_object> recs;
    for(const auto& b : m_Boundaries) recs.push_back(b.current);
    check(bnn_flip_set_boundaries(m_Gpu, recs.data(), (uint32_t)recs.size(), updateGrid ? 1 : 0),
          "bnn_flip_set_boundaries");
}

// PIC_Solver::advanceFrame (PIC_Solver.cpp:267-311): sub-steps until FrameDuration; the
// host vectors receive the particles at the end of the frame
void FLIP_GPU_Solver::advanceFrame() {
    FrameLog log;
    for(;;) {
        // PIC_Solver::advanceFrame (PIC_Solver.cpp:280-282) + advanceScene (:70-118): after
        // the first frame the dynamic objects move before every sub-step, and the boundary
        // SDF is recomputed when one of them did
        if(m_GlobalParams.finishedFrame > 0) {
            bool changed = false;
            const double fraction = (double)m_GlobalParams.frameLocalTime / (double)m_GlobalParams.frameDuration;
            for(auto& b : m_Boundaries)
                if(b.dynamic) changed |= b.update(m_GlobalParams.finishedFrame, fraction);
            if(changed) sendBoundaries(true);
        }
        bnn_step_stats st;
        const int rc = bnn_flip_step(m_Gpu, &st);
        check(rc, "bnn_flip_step");
        ++log.substeps;
        log.pcgIterations += st.pcg_iterations;
        log.lastResidual = st.pcg_residual;
        log.gpuMs += st.stage_ms[9];
        m_GlobalParams.frameLocalTime = (float)st.frame_time;
        if(st.frame_finished) break;
    }
    auto& D = m_ParticleData;
    check(bnn_flip_get_particles(m_Gpu, D.positions.data(), D.velocities.data()), "bnn_flip_get_particles");
    log.frame = m_GlobalParams.finishedFrame + 1;
    m_Logs.push_back(log);
}

// ParticleSolver::doFrameSimulation (ParticleSolver.cpp:160-186)
void FLIP_GPU_Solver::doFrameSimulation(unsigned frame) {
    (void)frame;
    advanceFrame();
    ++m_GlobalParams.finishedFrame;
    m_GlobalParams.frameLocalTime = 0.f;
    if(m_GlobalParams.bSaveFrameData) saveFrameData();
    if(m_GlobalParams.bSaveMemoryState) saveMemoryState();
}

// ParticleSolver::doSimulation (ParticleSolver.cpp:134-156); a resumed run continues
// after the frame of its memory state
void FLIP_GPU_Solver::doSimulation() {
    const unsigned first = std::max(m_GlobalParams.startFrame, m_GlobalParams.finishedFrame + 1u);
    for(unsigned frame = first; frame <= m_GlobalParams.finalFrame; ++frame) doFrameSimulation(frame);
    waitForFrameOutput();
}

void FLIP_GPU_Solver::finalizeSimulation() {
    waitForFrameOutput();
    if(m_Gpu) {
        bnn_flip_destroy(m_Gpu);
        m_Gpu = nullptr;
    }
}

void FLIP_GPU_Solver::waitForFrameOutput() {
    if(m_FrameWriter) {
        static_cast<std::future<void>*>(m_FrameWriter.get())->wait();
        m_FrameWriter.reset();
    }
}

// PIC_Solver::saveFrameData (PIC_Solver.cpp:236-263): particle_radius and compressed
// positions (the anisotropic kernel centres, with the kernel matrices, when "AniKernel"
// is asked for), plus object indices / compressed velocities when the scene asks for them;
// the file is written on a background thread while the next frame runs (the host arrays
// are copied first, so the caller may keep using them).
int FLIP_GPU_Solver::saveFrameData() {
    const auto& G = m_GlobalParams;
    if(!make_output_folder(G.dataPath, G.frameDataFolder)) return -1;
    auto file = std::make_shared<BnnFile>();
    const auto& D = m_ParticleData;
    file->nParticles = D.getNParticles();
    const float radius = m_SolverParams.particleRadius;
    file->setFixedReal("particle_radius", &radius, 1);
    if(G.savingData("ObjectIndex")) {
        file->setFixedUInt("NObjects", &D.nObjects, 1);
        std::vector<uint16_t> idx(D.objectIndex.begin(), D.objectIndex.end());
        file->setParticleUInt16("object_index", idx.data());
    }
    if(G.savingData("AniKernel")) {
        // AnisotropicKernelGenerator(positions, particleRadius) with its defaults; the
        // kernel centres replace the positions in the file (PIC_Solver.cpp:248-252)
        bnn_aniso_params ap;
        check(bnn_aniso_default_params(radius, &ap), "bnn_aniso_default_params");
        m_ParticleData.aniKernelCenters.resize(3 * (size_t)file->nParticles);
        m_ParticleData.aniKernelMatrices.resize(9 * (size_t)file->nParticles);
        check(bnn_flip_anisotropic_kernels(m_Gpu, &ap, m_ParticleData.aniKernelCenters.data(),
                                           m_ParticleData.aniKernelMatrices.data(), nullptr),
              "bnn_flip_anisotropic_kernels");
        file->setParticleCompressed("particle_position", D.aniKernelCenters.data(), 3);
        file->setParticleCompressedMatrix("anisotropic_kernel", D.aniKernelMatrices.data(), 3);
    } else {
        file->setParticleCompressed("particle_position", D.positions.data(), 3);
    }
    if(G.savingData("ParticleVelocity")) file->setParticleCompressed("particle_velocity", D.velocities.data(), 3);
    const std::string path = bnn_file_path(G.dataPath, G.frameDataFolder, "frame", (int)G.finishedFrame);
    waitForFrameOutput();
    auto fut = std::make_shared<std::future<void>>(std::async(std::launch::async, [file, path] { file->write(path); }));
    m_FrameWriter = std::static_pointer_cast<void>(fut);
    return 0;
}

// PIC_Solver::saveMemoryState (PIC_Solver.cpp:210-232): every FramePerState frames the
// grid resolution and face velocities, the particle radius, object count and the raw
// particle data
int FLIP_GPU_Solver::saveMemoryState() {
    const auto& G = m_GlobalParams;
    if(G.finishedFrame % G.framePerState != 0) return -1;
    if(!make_output_folder(G.dataPath, G.memoryStateDataFolder)) return -1;
    BnnFile file;
    int32_t gd[3];
    check(bnn_flip_grid_dims(m_Gpu, gd), "bnn_flip_grid_dims");
    const uint32_t res[3] = {(uint32_t)gd[0], (uint32_t)gd[1], (uint32_t)gd[2]};
    file.setFixedUInt("grid_resolution", res, 3);
    for(int d = 0; d < 3; ++d) {
        const size_t nf = (size_t)(res[0] + (d == 0)) * (res[1] + (d == 1)) * (res[2] + (d == 2));
        std::vector<float> u(nf);
        check(bnn_flip_get_grid(m_Gpu, d, u.data(), nf), "bnn_flip_get_grid");
        file.setFixedReal("grid_velocity_" + std::to_string(d), u.data(), (uint32_t)nf);
    }
    const auto& D = m_ParticleData;
    file.nParticles = D.getNParticles();
    file.setFixedUInt("NObjects", &D.nObjects, 1);
    const float radius = m_SolverParams.particleRadius;
    file.setFixedReal("particle_radius", &radius, 1);
    file.setParticleReal("particle_position", D.positions.data(), 3);
    file.setParticleReal("particle_velocity", D.velocities.data(), 3);
    std::vector<uint16_t> idx(D.objectIndex.begin(), D.objectIndex.end());
    file.setParticleUInt16("object_index", idx.data());
    return file.write(bnn_file_path(G.dataPath, G.memoryStateDataFolder, "frame", (int)G.finishedFrame)) ? 0 : -1;
}

// PIC_Solver::loadMemoryState (PIC_Solver.cpp:158-206): the latest state file up to
// FinalFrame; its particles and face velocities replace the generated ones
int FLIP_GPU_Solver::loadMemoryState() {
    const auto& G = m_GlobalParams;
    int frame = -1;
    BnnFile file;
    for(int f = (int)G.finalFrame; f >= 0; --f) {
        if(file.read(bnn_file_path(G.dataPath, G.memoryStateDataFolder, "frame", f))) {
            frame = f;
            break;
        }
    }
    if(frame < 0) return -1;
    std::vector<uint32_t> res;
    int32_t gd[3];
    check(bnn_flip_grid_dims(m_Gpu, gd), "bnn_flip_grid_dims");
    if(!file.getUInts("grid_resolution", res) || res.size() != 3 || (int)res[0] != gd[0] || (int)res[1] != gd[1] ||
       (int)res[2] != gd[2]) {
        std::fprintf(stderr, "%s: memory state grid does not match the scene\n", getSolverName().c_str());
        std::exit(EXIT_FAILURE);
    }
    auto& D = m_ParticleData;
    std::vector<float> pos, vel;
    if(!file.getFloats("particle_position", pos) || !file.getFloats("particle_velocity", vel) ||
       pos.size() != vel.size() || pos.size() != 3 * (size_t)file.nParticles) {
        std::fprintf(stderr, "%s: memory state without particle data\n", getSolverName().c_str());
        std::exit(EXIT_FAILURE);
    }
    D.positions = pos;
    D.velocities = vel;
    std::vector<uint16_t> idx;
    if(file.getUInt16("object_index", idx) && idx.size() == file.nParticles)
        D.objectIndex.assign(idx.begin(), idx.end());
    else
        D.objectIndex.assign(file.nParticles, 0);
    std::vector<uint32_t> nobj;
    if(file.getUInts("NObjects", nobj) && !nobj.empty()) D.nObjects = nobj[0];
    check(bnn_flip_set_particles(m_Gpu, D.positions.data(), D.velocities.data(), D.getNParticles()),
          "bnn_flip_set_particles");
    for(int d = 0; d < 3; ++d) {
        std::vector<float> u;
        if(!file.getFloats("grid_velocity_" + std::to_string(d), u)) std::exit(EXIT_FAILURE);
        check(bnn_flip_set_grid(m_Gpu, d, u.data(), u.size()), "bnn_flip_set_grid");
    }
    return frame;
}

} // namespace bnnhost
