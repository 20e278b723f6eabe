"""Copies the reference's shipped FLIP scene that the drop-in can run into
tests/golden/scenes/, with only "Solver" changed to the GPU solver's name.

Source: Applications/QtApps/ParticleSimulation/Scenes/FLIP3D_2DamBreak.json (two box
particle generators, CorrectPosition, AdvectionSteps 2).  The scene's other FLIP files use
a sphere particle generator (FLIP3D_BallDrop, FLIP3D_RotationalBoxBoundary, the latter also
an unregistered solver name), which the GPU solver's host class does not generate.

    python tests/golden/make_scene_fixtures.py <reference tree>
"""
import json
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit(f"usage: python {sys.argv[0]} <reference tree>")
src = Path(sys.argv[1]) / "Applications/QtApps/ParticleSimulation/Scenes/FLIP3D_2DamBreak.json"
scene = json.loads(src.read_text())
assert scene["GlobalParameters"]["Solver"] == "FLIP_3DSolver"
scene["GlobalParameters"]["Solver"] = "FLIP_GPU_3DSolver"
dst = Path(__file__).resolve().parent / "scenes" / "FLIP3D_2DamBreak.json"
dst.parent.mkdir(exist_ok=True)
dst.write_text(json.dumps(scene, indent=4) + "\n")
print(dst)
