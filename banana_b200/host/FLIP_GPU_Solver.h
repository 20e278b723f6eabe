// FLIP_GPU_Solver: the reference's ParticleSolver<3,float> plugin surface
// (Simulation/ParticleSolvers/ParticleSolver.h:39-105, FLIP_Solver.h) on top of the C ABI in
// banana_b200.h.  The public members keep the reference's names and meaning -- loadScene,
// doSimulation, doFrameSimulation, finalizeSimulation, globalParams, generalSolverParams,
// generalParticleData -- so a caller written against ParticleSolverInterface
// (Applications/QtApps/ParticleSimulation/Source/ParticleSolverInterface.h:55-173) works
// unchanged: after every frame the particle positions / velocities sit in host vectors of
// glm::vec3 layout (3 floats each) whose size never changes under the caller.
//
// Self-contained: it cannot include the reference headers here (their glm / json / spdlog
// submodules are not present), so parameters, particle data and the solver factory are
// small stand-ins with the reference's field names.  Inside the reference tree the class
// derives from FLIP_Solver<3,float> instead (see the integration notes).
#pragma once

#include <banana_b200.h>

#include "boundary_objects.h"

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace bnnhost {

struct Json;

// GlobalParameters (ParticleSolverData.h:37-75): the fields the FLIP sub-step reads
struct GlobalParameters {
    std::string solverName;
    float frameDuration = 1.0f / 30.0f;
    unsigned startFrame = 1u;
    unsigned finalFrame = 1u;
    unsigned finishedFrame = 0u;
    float frameLocalTime = 0.0f;
    bool bApplyGravity = true;
    bool bSaveFrameData = false;
    bool bSaveMemoryState = false;
    bool bLoadMemoryState = false;
    unsigned framePerState = 1u;
    std::string dataPath = ".";
    std::string frameDataFolder = "FrameData";
    std::string memoryStateDataFolder = "MemoryState";
    std::vector<std::string> SaveDataList;  // "OptionalSavingData": "ObjectIndex", "AniKernel", "ParticleVelocity"
    bool savingData(const std::string& name) const {
        for(const auto& s : SaveDataList)
            if(s == name) return true;
        return false;
    }
};

// SimulationParameters + PIC_Parameters (ParticleSolverData.h:87-175, PIC_Data.h:31-40),
// defaults from ParticleSolvers/Constants.h:31-54
struct SimulationParameters {
    float domainBMin[3] = {-1.f, -1.f, -1.f};
    float domainBMax[3] = {1.f, 1.f, 1.f};
    float movingBMin[3] = {-1.f, -1.f, -1.f};  // domain before padding (what the UI draws)
    float movingBMax[3] = {1.f, 1.f, 1.f};
    float cellSize = 1.0f / 64.0f;
    unsigned nExpandCells = 2u;
    float ratioCellSizePRadius = 2.0f;
    float particleRadius = 0.f;
    float minTimestep = 1.0e-6f;
    float maxTimestep = 1.0f / 30.0f;
    float CFLFactor = 1.0f;
    float CGRelativeTolerance = 1e-15f;
    unsigned maxCGIteration = 5000u;
    float PIC_FLIP_ratio = 0.97f;
    unsigned advectionSteps = 1u;
    bool bCorrectPosition = false;
    float repulsiveForceStiffness = 50.0f;
    bool bExitIfPressureProjectionFailed = false;
    unsigned maxNParticles = 0u;
    // GPU-only choices (no reference counterpart): precision of the pressure solve
    int pcgMode = BNN_PCG_FP32;
    float refineTolerance = 1e-8f;
    float refineInnerTolerance = 1e-2f;  // measured best at 256^3 (1e-3: 0.69 G, 1e-2: 0.72 G particle-steps/s)
};

// ParticleSimulationData (ParticleSolverData.h:178-241): AoS vec3 host arrays
struct ParticleData {
    std::vector<float> positions;   // 3 floats per particle
    std::vector<float> velocities;  // 3 floats per particle
    std::vector<int16_t> objectIndex;
    unsigned nObjects = 0;
    // anisotropic kernels of the last saved frame (3 floats / 9 floats column-major each)
    std::vector<float> aniKernelCenters;
    std::vector<float> aniKernelMatrices;
    unsigned getNParticles() const { return (unsigned)(positions.size() / 3); }
};

// Per-frame record (what the reference's logger prints per sub-step / frame)
struct FrameLog {
    unsigned frame = 0;
    unsigned substeps = 0;
    unsigned pcgIterations = 0;     // summed over the frame's sub-steps
    double lastResidual = 0.0;
    float gpuMs = 0.f;              // summed stage_ms[9] of the sub-steps
};

class FLIP_GPU_Solver {
public:
    static constexpr int dimension() noexcept { return 3; }
    static std::string solverName() { return "FLIP_GPU_3DSolver"; }
    static std::shared_ptr<FLIP_GPU_Solver> createSolver() { return std::make_shared<FLIP_GPU_Solver>(); }

    explicit FLIP_GPU_Solver(int solverKind = BNN_SOLVER_FLIP) : m_SolverKind(solverKind) {}
    virtual ~FLIP_GPU_Solver();
    FLIP_GPU_Solver(const FLIP_GPU_Solver&) = delete;
    FLIP_GPU_Solver& operator=(const FLIP_GPU_Solver&) = delete;

    // ParticleSolver public API (ParticleSolver.cpp:36-238).  A scene with LoadMemoryState
    // resumes from the latest state file; doSimulation then continues after that frame.
    // allocate = false stops after the particles are generated (no GPU needed)
    void loadScene(const std::string& sceneFile, bool allocate = true);
    void loadSceneFromString(const std::string& sceneJson, bool allocate = true);
    void doSimulation();
    void doFrameSimulation(unsigned frame);
    void finalizeSimulation();

    virtual std::string getSolverName() { return solverName(); }
    virtual std::string getSolverDescription() { return "Simulation using FLIP-3D Solver on a B200 GPU"; }

    GlobalParameters& globalParams() noexcept { return m_GlobalParams; }
    SimulationParameters& generalSolverParams() noexcept { return m_SolverParams; }
    ParticleData& generalParticleData() noexcept { return m_ParticleData; }

    // GPU-side extras
    const std::vector<FrameLog>& frameLogs() const { return m_Logs; }
    bnn_flip* handle() { return m_Gpu; }
    // Replace the generated particles (before the first frame), e.g. with a saved state
    void setParticles(const std::vector<float>& pos, const std::vector<float>& vel);

protected:
    // ParticleSolver / PIC_Solver protected virtuals (ParticleSolver.h:70-92)
    virtual void generateParticles(const Json& scene);
    virtual void allocateSolverMemory();
    virtual void advanceFrame();
    virtual void sortParticles() {}  // the device sorts by cell every sub-step
    // .bnn frame output and memory states (PIC_Solver.cpp:123-263); 0 = done, -1 = not
    // done / failed; loadMemoryState returns the frame of the state it loaded
    virtual int saveFrameData();
    virtual int saveMemoryState();
    virtual int loadMemoryState();
    void waitForFrameOutput();

    // A failing C ABI call: log it, and exit where the reference exits (__BNN_REQUIRE,
    // Macros.h:225-233; ExitIfPressureProjectionFailed, PIC_Solver.cpp:901-906)
    void check(int status, const char* what);

    int m_SolverKind;
    double m_CellSizeScene = 1.0 / 64.0;  // CellSize as written in the scene (the sampler's grid)
    GlobalParameters m_GlobalParams;
    SimulationParameters m_SolverParams;
    ParticleData m_ParticleData;
    bnn_flip* m_Gpu = nullptr;
    std::vector<FrameLog> m_Logs;
    // "AdditionalBoundaryObjects" of the scene and their current transformations
    std::vector<BoundaryObjectSpec> m_Boundaries;
    void sendBoundaries(bool updateGrid);
    std::shared_ptr<void> m_FrameWriter;  // std::future of the frame file being written
};

class APIC_GPU_Solver : public FLIP_GPU_Solver {
public:
    APIC_GPU_Solver() : FLIP_GPU_Solver(BNN_SOLVER_APIC) {}
    static std::string solverName() { return "APIC_GPU_3DSolver"; }
    std::string getSolverName() override { return solverName(); }
};

class AFLIP_GPU_Solver : public FLIP_GPU_Solver {
public:
    AFLIP_GPU_Solver() : FLIP_GPU_Solver(BNN_SOLVER_AFLIP) {}
    static std::string solverName() { return "AFLIP_GPU_3DSolver"; }
    std::string getSolverName() override { return solverName(); }
};

class PIC_GPU_Solver : public FLIP_GPU_Solver {
public:
    PIC_GPU_Solver() : FLIP_GPU_Solver(BNN_SOLVER_PIC) {}
    static std::string solverName() { return "PIC_GPU_3DSolver"; }
    std::string getSolverName() override { return solverName(); }
};

// ParticleSolverFactory (ParticleSolverFactory.h:30-60): solvers by name, and by the
// "Solver" entry of a scene's GlobalParameters
class ParticleSolverFactory {
public:
    using CreateMethod = std::function<std::shared_ptr<FLIP_GPU_Solver>()>;
    static bool registerSolver(const std::string& name, CreateMethod create);
    static std::shared_ptr<FLIP_GPU_Solver> createSolver(const std::string& name);
    static std::shared_ptr<FLIP_GPU_Solver> createSolverFromJSon(const std::string& sceneFile);

private:
    static std::map<std::string, CreateMethod>& methods();
};

// Seeded particle sampling of a box generator (replaces ParticleGenerator's
// process-global MT jitter, ParticleGenerator.cpp:97-114): every grid cell lying fully
// inside [bmin, bmax] gets `ppc` particles, uniform in the cell, from SplitMix64 over
// (seed, axis, cell * ppc + k).  Appends AoS positions and zero velocities.
void sample_box(const float domainMin[3], double cellSize, const double bmin[3], const double bmax[3], unsigned ppc,
                uint64_t seed, std::vector<float>& pos, std::vector<float>& vel);

} // namespace bnnhost
