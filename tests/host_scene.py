"""Scene JSON for the host C++ driver tests: the dam break of banana_b200.scenes written
the way the reference's scene files are (GlobalParameters / SimulationParameters /
ParticleGenerators)."""
import json

import numpy as np


def dam_break_scene(n: int, frames: int = 2, block=(0.4, 0.6, 0.4), solver: str = "FLIP_GPU_3DSolver",
                    **globals_) -> str:
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    g = {"Solver": solver, "FrameDuration": f32(1.0 / 30.0), "StartFrame": 1, "FinalFrame": frames,
         "SaveFrameData": False}
    g.update(globals_)
    return json.dumps({
        "GlobalParameters": g,
        "SimulationParameters": {
            "SimulationDomainBox": {"BoxMin": [0, 0, 0], "BoxMax": [1, 1, 1]},
            "CellSize": 1.0 / n, "NExpandCells": 2, "CFLFactor": 1, "MinTimestep": 1e-6,
            "MaxTimestep": f32(np.float32(1.0) / np.float32(30.0)), "PIC_FLIP_ratio": 0.97,
            "CGRelativeTolerance": 1e-6, "MaxCGIteration": 5000, "AdvectionSteps": 1},
        "ParticleGenerators": [{"GeometryType": "Box", "UniqueName": "Dam", "BoxMin": [0, 0, 0],
                                "BoxMax": list(block), "ParticlesPerCell": 8, "Seed": 42}],
    }, indent=1)


def read_particles(path):
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:4], np.uint32)[0])
    a = np.frombuffer(raw[4:], np.float32)
    return a[:3 * n].reshape(n, 3), a[3 * n:6 * n].reshape(n, 3)
