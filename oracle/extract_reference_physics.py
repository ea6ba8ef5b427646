"""TEST INFRASTRUCTURE (oracle build step): extracts, unchanged, the member
functions of the reference's CPU steps (src/cpu/UnifiedPhysics.cpp) that the
PCISPH coupling step with static boundaries and rigid bodies and the WCSPH
step run, so that oracle/Makefile can compile
them beside a minimal class declaration of its own (ref_physics_harness.h)
instead of the whole translation unit, whose includes need a graphics
stack. The output goes to oracle/_ref/ only (never committed).

    python extract_reference_physics.py <reference UnifiedPhysics.cpp> <output .cpp>
"""
import re
import sys

# CpuParticlePhysicsVersatileCouplingPCISPH (UnifiedPhysics.cpp:4991-5024)
# and every member function it reaches on a scene of liquid and frozen
# boundary particles, plus the weighted boundary volume of set-up
FUNCTIONS = [
    "CpuParticlePhysicsVersatileCouplingPCISPH",
    "NeighborSearchOMP", "GetNeighbors",
    "CalculateWeightedVolumeOMP", "CalculateWeightedVolume",
    "CalculateExternalForcesVersatilCouplingPCISPHOMP", "CalculateExternalForcesVersatilCouplingPCISPH",
    "CalculateBoundaryFluidPressureForceHost", "CalculateSurfaceTensionForcePCISPHHost",
    "CalculateSurfaceCohesionForcePCISPHHost", "CalculateSpringForceHost", "CalculateDampingForceHost",
    "CalculateBoundaryForcePerLiquidParticleHost", "CalculateBoundaryForcePerRigidParticleHost", "BoxBoundaryForce",
    "PredictionCorrectionStep", "PredictPositionAndVelocity", "CollisionHandling",
    "ComputePredictedDensityAndPressure", "ComputeCorrectivePressureForce",
    "UpdateLiquidParticlePosVelSphCPUOMP", "UpdateLiquidParticlePosVelSphCPU",
    "BoundaryHandlingPureFluidOMP", "BoundaryHandlingBoxPerNonRigidParticle",
    "SortParticles",
    "RigidBodyIntegrationOMP", "UpdateRigidBodyParticleInformationOMP", "SynRigidParticlesOMP",
]
# CpuParticlePhysicsPureFluidsSPH (the WCSPH step, UnifiedPhysics.cpp:4200-4260)
# and what it calls beyond the functions above
FUNCTIONS += [
    "CpuParticlePhysicsPureFluidsSPH", "CalculateDensityPressurePureFluidSPH", "CalculatePressureSPH",
    "CalculatePressureWCSPH", "CalculateLiquidParticleForces", "CalculateSurfaceTensionForcePCISPH",
    "DistanceToWall", "WallWeight",
]
# The per-body functions of the rigid phase (force and torque sums and the
# body update, the particle sync) and AddToRigidBody, with which the pin's
# set-up assembles bodies as the reference's scene construction does, one
# particle at a time. CalculateRigidBodyForceTorqueMomenta's old-method branch
# binds a temporary to a non-const reference (an MSVC extension);
# ref_physics_harness.h gives GCC an overload that makes the same call on a
# copy.
FUNCTIONS += ["CalculateRigidBodyForceTorqueMomenta", "SynRigidParticlesPerRigidBody", "AddToRigidBody"]


def definition(src, name):
    """The text of `... UnifiedPhysics::name(...) { ... }` (first definition)."""
    m = re.search(r"^[^\n;{}]*\bUnifiedPhysics::" + name + r"\s*\(", src, re.M)
    if not m:
        raise SystemExit("definition of UnifiedPhysics::%s not found" % name)
    start = m.start()
    brace = src.index("{", m.end())
    depth, k = 0, brace
    while True:
        c = src[k]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                break
        k += 1
    line = src.count("\n", 0, start) + 1
    return "#line %d \"UnifiedPhysics.cpp\"\n" % line + src[start:k + 1] + "\n"


def quicksort_pointer(src):
    """The file-scope QuickSort function pointer the range sort calls."""
    m = re.search(r"^void \(\*QuickSort\)\(.*?>;\s*$", src, re.M | re.S)
    if not m:
        raise SystemExit("QuickSort definition not found")
    return src[m.start():m.end()] + "\n"


def main():
    src = open(sys.argv[1], encoding="utf-8-sig", errors="replace").read().replace("\r\n", "\n")
    out = ['#include "ref_physics_harness.h"\n', quicksort_pointer(src)]
    out += [definition(src, f) for f in FUNCTIONS]
    open(sys.argv[2], "w").write("\n".join(out))


if __name__ == "__main__":
    main()
