#!/usr/bin/env python
"""Benchmark of the per-step particle pipeline.

Workload (N=1): PCISPH dam break, 128^3 = 1,048,576 fluid particles
(spacing 0.01, jitter +-0.001) in a 2 x 1.3 x 1.3 container with two shells
of boundary particles (~276k), h = 0.02, 1% density error, 3-50
predict-correct iterations, dt = 5e-4, full Morton sort every step.
Metric: fluid particle-steps per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--scene c2|c2-small|c1|c3]

--scene c3 times the rigid-fluid coupling workload instead: 524,288 PCISPH
fluid particles, a 131,072-grain granular pile (friction 0.5) and 16 rigid
bodies (spheres, cubes, tori, radii 0.05-0.15, 2k-8k surface particles each);
its metric counts every dynamic particle (fluid, grains, rigid).

One JSON line on rank 0. Under torchrun (N > 1) every rank runs its own
replica of the scene (the single-scene path does not shard: replicas only),
value = all ranks' particle-steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from unifiedparticleframeworkcuda_b200 import replicas  # noqa: E402

METRIC = "particle-steps/s at 1M PCISPH (<1% density err)"
UNIT = "particle-steps/s"
RADIX_PASSES = 4  # 30-bit Morton keys, 8-bit digits


def scene_for(args):
    from unifiedparticleframeworkcuda_b200 import scenes
    if args.scene == "c2":
        return scenes.pcisph_dam(128, 128, 64)
    if args.scene == "c2-small":
        return scenes.pcisph_dam(64, 64, 64)
    if args.scene == "c1":
        sc = scenes.wcsph_dam(32)
        sc.params.dt = C1_DT
        return sc
    if args.scene == "c3":
        return scenes.coupling_scene()
    raise SystemExit("unknown scene " + args.scene)


# The WCSPH dam at its specified dt = 1e-3 diverges within 12 steps in the
# reference's own WCSPH method (the oracle's kinetic energy goes from 317 J to
# 4.5e6 J: the step is twice the sound-speed limit 0.4 h / c with c =
# sqrt(gamma B / rho0) = 31.6 m/s). The timed line runs at half that step,
# which stays bounded over 300 steps; everything else is as specified.
C1_DT = 5e-4
C1_NOTE = "dt halved from the specified 1e-3, which diverges within 12 steps in the reference's own WCSPH method"


def cpu_sample_scene(args):
    """The bounded CPU sample of a workload: same physics, fewer particles."""
    from unifiedparticleframeworkcuda_b200 import scenes
    if args.scene == "c3":
        return scenes.coupling_scene(fluid=(64, 32, 32), granular=(32, 16, 32), n_bodies=4), \
            "coupling 64x32x32 fluid + 32x16x32 grains + 4 bodies"
    if args.scene == "c1":
        return scene_for(args), "wcsph_dam 32^3 (the workload itself)"
    return scenes.pcisph_dam(64, 64, 64), "pcisph_dam 64^3"


# Steps from rest after which the dam's predict-correct loop meets the 1%
# density error criterion. Measured on the 1M dam (per-step trace over 8,000
# steps): steps 0-43 (the jittered lattice's start-up transient) end at the
# 50-iteration cap with errors of 1-11%; steps 44-274 all end below 1%
# (7-35 iterations) while the column collapses; from about step 275 the
# surges against the walls send 20-60% of the steps back to the cap. The
# timed steps (both arms) start from the state after these steps, so that a
# default run (settle + warm-up + timed steps within 224 steps) times steps
# that meet the criterion.
SETTLE_DEFAULT = {"c2": 50, "c2-small": 50}


def settle_steps(args):
    return SETTLE_DEFAULT.get(args.scene, 0) if args.settle < 0 else args.settle


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def state_of_system(s, sc):
    """System `s`'s current state (the workload `sc` advanced on the GPU) per
    input particle: positions, velocities, and the lagged PCISPH state (the
    step before last's and the last step's correction pressures, the last
    predicted density) of the dynamic particles, the boundary as built.
    Returns (params, pos, vel, (prev, pressure, density))."""
    import unifiedparticleframeworkcuda_b200 as upf
    g = s.particles()
    lag = s.lagged_state()  # (previous correction pressure, last one, last predicted density), same order
    ids = g["id"].astype(np.int64)
    pos = np.array(sc.pos, np.float32, copy=True)
    vel = np.array(sc.vel, np.float32, copy=True)
    p = upf.derive_params(sc.params)
    prev = np.zeros(sc.n, np.float32)
    pres = np.zeros(sc.n, np.float32)
    dens = np.full(sc.n, np.float32(p.rest_density), np.float32)
    pos[ids] = g["pos"]
    vel[ids] = g["vel"]
    prev[ids] = lag[:, 0]
    pres[ids] = lag[:, 1]
    dens[ids] = lag[:, 2]
    return p, pos, vel, (prev, pres, dens)


def oracle_from_system(s, sc, threads, fp64=False):
    """The oracle (FP32, or its FP64 twin) holding system `s`'s current state
    (state_of_system)."""
    from oracle import pyoracle
    p, pos, vel, lag = state_of_system(s, sc)
    o = pyoracle.OracleSim(p, pos, vel, sc.type, threads=threads, keep_fields=False, fp64=fp64)
    o.set_lagged(*lag)
    return o


# Workloads whose CPU legs time the reference's own step: its
# CpuParticlePhysicsVersatileCouplingPCISPH / CpuParticlePhysicsPureFluidsSPH
# (src/cpu/UnifiedPhysics.cpp) compiled from its sources into
# oracle/_ref/libupfref_physics.so by oracle/Makefile (oracle/refstep.py).
# The coupling workload keeps the oracle: its granular pile is not part of
# the reference's coupling step.
REFERENCE_STEP_SCENES = {"c2": "pcisph", "c2-small": "pcisph", "c1": "wcsph"}


def reference_step_available(args):
    if args.scene not in REFERENCE_STEP_SCENES:
        return False
    from oracle import refstep
    return refstep.available()


def time_reference_step(args, p, sc, pos, vel, lagged, threads, warmup, steps, min_steps, max_seconds):
    """The reference's step on the host cores from the given state; returns
    (particle-steps/s, timed steps, mean iterations, steps at the cap, largest
    final density error in percent, seconds)."""
    from oracle import refstep
    r = refstep.reference_time(p, pos, vel, sc.type, lagged, REFERENCE_STEP_SCENES[args.scene], threads=threads,
                               warmup=warmup, steps=steps, max_seconds=max_seconds, min_steps=min_steps)
    secs = float(r["seconds"].sum())
    done = int(r["seconds"].size)
    its = r["iterations"]
    return (dynamic_count(sc) * done / secs, done, float(its.mean()), int((its >= p.max_loops).sum()),
            float(r["error_percent"].max()), secs)


def fp64_error(s, sc, threads):
    """One step of system `s` from its checkpoint 0 (the state at the start
    of the timed steps) against the FP64 oracle from the same state: the
    largest differences of the liquid particles' fields (positions absolute
    in m, the rest relative to the field's largest magnitude) and both
    iteration counts (0 for WCSPH)."""
    import unifiedparticleframeworkcuda_b200 as upf
    s.restore(0)
    o = oracle_from_system(s, sc, threads, fp64=True)
    if sc.num_bodies:
        # bodies assembled from their particles' current positions and
        # velocities (FP64 sums on both sides)
        o.set_rigid_bodies(sc.body, sc.num_bodies)
    s.step(1)
    s.synchronize()
    gi = s.stats().iterations
    g = s.particles()
    info = o.step()
    c = o.state()
    o.close()
    liq = np.sort(g["id"][g["type"] == upf.LIQUID])
    out = {"iterations_gpu": int(gi), "iterations_fp64": int(info.iterations)}
    go, co = np.argsort(g["id"]), np.argsort(c["id"])
    gs = go[np.searchsorted(g["id"][go], liq)]
    cs = co[np.searchsorted(c["id"][co], liq)]
    for k in ("pos", "vel", "density", "pressure"):
        a = g[k][gs].astype(np.float64)
        b = c[k][cs].astype(np.float64)
        if a.ndim == 2:
            a, b = a[:, :3], b[:, :3]
        scale = 1.0 if k == "pos" else max(np.abs(b).max(), 1e-30)
        out[("pos_max_abs_m" if k == "pos" else k + "_max_rel")] = float(np.abs(a - b).max() / scale)
    return out


def workload_name(args):
    return {"c2": "pcisph_dam_break_1M", "c2-small": "pcisph_dam_break_262k",
            "c1": "wcsph_dam_break_32k", "c3": "rigid_fluid_granular_coupling_524k"}[args.scene]


def metric_for(args):
    if args.scene == "c3":
        return "particle-steps/s, rigid-fluid coupling + granular (524k fluid, 131k grains, 16 bodies)"
    if args.scene == "c1":
        return "particle-steps/s, WCSPH dam break (32,768 fluid, h=0.04, dt=5e-4)"
    return METRIC


def dynamic_count(sc):
    return sc.n - sc.n_boundary


def algorithmic_bytes(nf, nb, steps, total_iters, method):
    """Algorithmic HBM bytes of `steps` steps: every SoA array counted once per
    pass, neighbour re-reads counted zero. PCISPH: N_f (241 + 20P + 112 k) +
    N_b 20 (1 + 2k) per step; WCSPH: N_f (193 + 20P) + N_b 40."""
    if method == "pcisph":
        return steps * (nf * (241 + 20 * RADIX_PASSES) + nb * 20) + total_iters * (112 * nf + 40 * nb)
    return steps * (nf * (193 + 20 * RADIX_PASSES) + nb * 40)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 7 and f[0].replace(".", "").isdigit():
                    rows.append(f)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[2]) for r in rows)}


def make_oracle(sc, threads):
    from oracle import pyoracle
    import unifiedparticleframeworkcuda_b200 as upf
    p = upf.derive_params(sc.params)
    o = pyoracle.OracleSim(p, sc.pos, sc.vel, sc.type, threads=threads, keep_fields=False)
    if sc.num_bodies:
        o.set_rigid_bodies(sc.body, sc.num_bodies)
    return o


def full_config_oracle(args, threads):
    """The dam workload at its full size for the reference arm: the oracle
    advanced from rest by the workload's settle steps on the host cores (the
    same procedure the GPU arm runs before its timed steps). Returns
    (oracle, scene, label, settle info)."""
    sc = scene_for(args)
    settle = settle_steps(args)
    o = make_oracle(sc, threads)
    t0 = time.perf_counter()
    its = [o.step().iterations for _ in range(settle)]
    info = {"settle_steps": settle, "settle_seconds": time.perf_counter() - t0,
            "settle_mean_iterations": float(np.mean(its)) if its else 0.0}
    label = "%s after %d steps from rest" % (workload_name(args), settle) if settle else \
        "%s from rest" % workload_name(args)
    return o, sc, label, info


def cpu_baseline(args, seconds=15.0, system=None):
    """The CPU baseline on the host cores: the reference's own step where it
    covers the workload (REFERENCE_STEP_SCENES, kind "reference"), else the
    oracle (the FP32 OpenMP restatement of the reference CPU path, kind
    "port"). Given the GPU arm's system (the dam workloads), it runs the full
    configuration from that system's state: 2 warm-up steps, then steps
    until at least 5 and `seconds` have passed. The other workloads run the
    workload itself (WCSPH) or a bounded sample of the same scene (the same
    spacing, h, dt and boundary with fewer particles)."""
    from oracle import pyoracle
    pyoracle.build(with_ref=False)
    threads = os.cpu_count() or 1
    if reference_step_available(args):
        # the reference's own step: from the GPU arm's state at the start of
        # its timed steps (the dams), or the workload itself from rest
        sc = scene_for(args)
        if system is not None:
            p, pos, vel, lag = state_of_system(system, sc)
            label = "%s after %d steps from rest, the state the GPU arm times" % (workload_name(args),
                                                                                 settle_steps(args))
            warm, min_steps = 2, 5
        else:
            import unifiedparticleframeworkcuda_b200 as upf
            p, pos, vel, lag = upf.derive_params(sc.params), sc.pos, sc.vel, None
            label = "%s from rest" % workload_name(args)
            warm, min_steps = 1, 2
        v, done, mean_its, _, _, secs = time_reference_step(args, p, sc, pos, vel, lag, threads, warm, 100000,
                                                            min_steps, seconds)
        return {"value": v, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "reference",
                "sample": "the reference's own step (src/cpu/UnifiedPhysics.cpp, compiled from its sources, %d "
                          "OpenMP threads) on %d dynamic + %d boundary particles (%s), %d steps after %d warm-up, "
                          "mean %.1f iterations, %.1f s" % (threads, dynamic_count(sc), sc.n_boundary, label, done,
                                                            warm, mean_its, secs)}
    if system is not None:
        # the full configuration from the GPU arm's own state at the start of
        # its timed steps
        sc = scene_for(args)
        o = oracle_from_system(system, sc, threads)
        label = "%s after %d steps from rest, the state the GPU arm times" % (workload_name(args),
                                                                             settle_steps(args))
        warm, min_steps = 2, 5
    else:
        sc, label = cpu_sample_scene(args)
        o = make_oracle(sc, threads)
        warm, min_steps = 1, 2
    for _ in range(warm):
        o.step()
    t0 = time.perf_counter()
    steps = 0
    iters = 0
    while True:
        info = o.step()
        steps += 1
        iters += info.iterations
        if time.perf_counter() - t0 >= seconds and steps >= min_steps:
            break
    dt = time.perf_counter() - t0
    o.close()
    nd = dynamic_count(sc)
    return {"value": nd * steps / dt, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
            "sample": "%d dynamic + %d boundary particles (%s), %d steps after %d warm-up, mean %.1f iterations, "
                      "%.1f s" % (nd, sc.n_boundary, label, steps, warm, iters / steps, dt)}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU step on the host cores. The dam
    and WCSPH workloads run the reference's own step functions, compiled
    from its sources (oracle/_ref/libupfref_physics.so); the others, and a
    checkout without the compiled reference, run the oracle port."""
    if rank != 0:
        return
    if args.scene == "c4":
        from unifiedparticleframeworkcuda_b200 import scenes
        cb = batch_cpu_baseline(scenes.batch_scenes(args.batch_scenes), args.cpu_seconds)
        print(json.dumps({
            "impl": "reference", "metric": "batched scene-steps/s (256 PCISPH scenes, 2k-65k particles) vs "
                                          "sequential single-scene steps",
            "value": cb["value"], "unit": cb["unit"], "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / cb["value"] * args.batch_scenes, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched_pcisph_256_scenes"}, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return
    if args.scene == "io":
        run_io_reference(args)
        return
    if args.scene == "mesh":
        tri, _ = mesh_workload()
        cb = mesh_reference_sample(tri)
        base = {"impl": "reference", "metric": MESH_METRIC, "unit": "point-face tests/s"}
        if cb is None:
            print(json.dumps(dict(base, unavailable="oracle/_ref/libupfref.so (the compiled reference loader) is "
                                                    "not built")), flush=True)
            return
        print(json.dumps(dict(base, value=cb["value"], n_gpus=args.gpus, steps=1, warmup=0, higher_is_better=True,
                              scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                              config={"workload": "icosphere_5120_faces_2mm"}, cpu_baseline=cb,
                              e2e={"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0,
                                   "d2h_bytes_per_step": 0})), flush=True)
        return
    from oracle import pyoracle
    pyoracle.build(with_ref=False)
    threads = os.cpu_count() or 1
    full = args.scene in ("c2", "c2-small")
    if reference_step_available(args):
        run_reference_step(args, threads, full)
        return
    if full:
        # the full configuration, advanced by the same settle steps as the
        # GPU arm before its timed steps
        o, sc, label, settle_info = full_config_oracle(args, threads)
    else:
        # bounded sample per step: a smaller block of the workload
        sc, label = cpu_sample_scene(args)
        o = make_oracle(sc, threads)
    for _ in range(args.warmup):
        o.step()
    t0 = time.perf_counter()
    iters = 0
    at_max = 0
    max_err = 0.0
    p = o.params
    for _ in range(args.steps):
        info = o.step()
        iters += info.iterations
        at_max += int(info.iterations >= p.max_loops)
        max_err = max(max_err, float(info.density_error_percent))
    dt = time.perf_counter() - t0
    o.close()
    v = dynamic_count(sc) * args.steps / dt
    cfg = {"workload": workload_name(args), "mean_iterations": iters / max(args.steps, 1),
           **({"dt": C1_DT, "dt_note": C1_NOTE} if args.scene == "c1" else {})}
    if full:
        cfg.update({"fluid_particles": sc.n_fluid, "boundary_particles": sc.n_boundary, **settle_info,
                    "state": label, "steps_at_max_loops": at_max,
                    "max_step_density_error_percent": max_err, "same_config": True})
    else:
        cfg.update({"sample_fluid_particles": sc.n_fluid, "sample_boundary_particles": sc.n_boundary,
                    "same_config": False})
    print(json.dumps({
        "impl": "reference", "metric": metric_for(args), "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
                         "sample": "%s: %d dynamic + %d boundary per step" % (label, dynamic_count(sc),
                                                                              sc.n_boundary)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_reference_step(args, threads, full):
    """The reference arm on the reference's own step. The dams: the full
    configuration advanced from rest by the workload's settle steps (by the
    oracle, as in the other arms' CPU legs: the reference's own settle steps,
    most of them at the 50-iteration cap, would take the 1M scene several
    minutes of host time), handed over with its lagged PCISPH state, then the
    reference's warm-up and timed steps: `--steps` of them, or as many as
    `--ref-seconds` allow (at least 3). WCSPH: the workload from rest."""
    import unifiedparticleframeworkcuda_b200 as upf
    if full:
        o, sc, label, settle_info = full_config_oracle(args, threads)
        st = o.state()
        lag = o.lagged()
        o.close()
        order = np.argsort(st["id"])
        p = upf.derive_params(sc.params)
        pos, vel = st["pos"][order], st["vel"][order]
        label += " (settled by the oracle)"
    else:
        sc = scene_for(args)
        p = upf.derive_params(sc.params)
        pos, vel, lag, settle_info = sc.pos, sc.vel, None, {}
        label = "%s from rest" % workload_name(args)
    warm = min(args.warmup, 2) if full else args.warmup
    v, done, mean_its, at_max, max_err, secs = time_reference_step(
        args, p, sc, pos, vel, lag, threads, warm, args.steps, min(args.steps, 3), args.ref_seconds)
    cfg = {"workload": workload_name(args), "fluid_particles": sc.n_fluid, "boundary_particles": sc.n_boundary,
           **settle_info, "state": label, "timed_steps": done, "same_config": True,
           **({"dt": C1_DT, "dt_note": C1_NOTE} if args.scene == "c1" else {})}
    if REFERENCE_STEP_SCENES[args.scene] == "pcisph":
        cfg.update({"mean_iterations": mean_its, "steps_at_max_loops": at_max,
                    "max_step_density_error_percent": max_err})
    sample = ("the reference's own step (src/cpu/UnifiedPhysics.cpp, compiled from its sources, %d OpenMP "
              "threads): %d dynamic + %d boundary particles, %s; %d timed steps of the %d requested after %d "
              "warm-up (bounded to %.0f s), %.1f s" % (threads, dynamic_count(sc), sc.n_boundary, label, done,
                                                        args.steps, warm, args.ref_seconds, secs))
    print(json.dumps({
        "impl": "reference", "metric": metric_for(args), "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "reference",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def batch_cpu_baseline(scs, seconds):
    """A bounded sample of the batch (every 64th scene) on the host cores,
    as particle-steps/s converted to scene-steps/s by the batch's mean scene
    size: the reference's own step (each scene in its own process, from rest,
    an even share of `seconds` each) where it is compiled, else the oracle."""
    from oracle import pyoracle, refstep
    pyoracle.build(with_ref=False)
    threads = os.cpu_count() or 1
    sample = scs[::64]
    if refstep.available():
        import unifiedparticleframeworkcuda_b200 as upf
        parts, steps_total, secs = 0, 0, 0.0
        for sc in sample:
            p = upf.derive_params(sc.params)
            r = refstep.reference_time(p, sc.pos, sc.vel, sc.type, None, "pcisph", threads=threads, warmup=1,
                                       steps=100000, max_seconds=seconds / len(sample), min_steps=2)
            parts += sc.n * r["seconds"].size
            steps_total += r["seconds"].size
            secs += float(r["seconds"].sum())
        pps = parts / secs
        mean_n = sum(sc.n for sc in scs) / len(scs)
        return {"value": pps / mean_n, "unit": "scene-steps/s", "cores": threads, "kind": "reference",
                "cpu_model": cpu_model(),
                "sample": "the reference's own step (src/cpu/UnifiedPhysics.cpp, compiled from its sources, %d "
                          "OpenMP threads) on %d of %d scenes (%d particles) from rest, each in its own process, "
                          "%d steps in all after one warm-up each, %.1f s: %.3g particle-steps/s over the batch's "
                          "mean scene size %.0f" % (threads, len(sample), len(scs), sum(sc.n for sc in sample),
                                                    steps_total, secs, pps, mean_n)}
    sims = [make_oracle(sc, threads) for sc in sample]
    for o in sims:
        o.step()
    t0 = time.perf_counter()
    steps = 0
    while True:
        for o in sims:
            o.step()
        steps += 1
        if time.perf_counter() - t0 >= seconds and steps >= 2:
            break
    dt = time.perf_counter() - t0
    for o in sims:
        o.close()
    nsample = sum(sc.n for sc in sample)
    pps = nsample * steps / dt
    mean_n = sum(sc.n for sc in scs) / len(scs)
    return {"value": pps / mean_n, "unit": "scene-steps/s", "cores": threads, "kind": "port",
            "sample": "%d of %d scenes (%d particles), %d steps, %.1f s: %.3g particle-steps/s over the batch's "
                      "mean scene size %.0f" % (len(sample), len(scs), nsample, steps, dt, pps, mean_n)}


def run_batch(args, rank, world, local_rank):
    """--scene c4: the batched form. 256 scenes (log-uniform 2,048-65,536
    particles, box extents U(0.5, 2.0)) advance together; the baseline is the
    same scenes as 256 single-scene systems stepped one after another."""
    import ctypes as C

    import torch
    import unifiedparticleframeworkcuda_b200 as upf
    from unifiedparticleframeworkcuda_b200 import build as upfbuild
    from unifiedparticleframeworkcuda_b200 import scenes

    if rank == 0:
        upfbuild.build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    scs = scenes.batch_scenes(args.batch_scenes, seed=2024 + rank)
    ns = len(scs)
    npart = sum(sc.n for sc in scs)
    stream = torch.cuda.Stream(device=dev)
    b = upf.ParticleBatch.from_scenes(scs, device=local_rank)
    b.set_stream(stream.cuda_stream)
    b.step(args.warmup)
    b.synchronize()
    if args.shape:
        b.set_launch_config(parse_shape(args.shape))
        tuned = b.launch_config().as_dict()
    else:
        tuned = b.autotune(3).as_dict() if not args.no_autotune else b.launch_config().as_dict()
    b.reset_counters()
    b.checkpoint(0)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def timed(fn, clk=None):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return replicas.max_over_ranks(e0.elapsed_time(e1))[0]

    with ClockSampler(local_rank) as clk:
        batch_ms = timed(lambda: b.step(args.steps))
    b.synchronize()
    stats = b.stats()
    its = [st.total_iterations / max(st.total_steps, 1) for st in stats]
    errs = [st.density_error_percent for st in stats]
    value = ns * args.steps * world / (batch_ms / 1e3)

    # per-pass timings of one step (dominant kernel: the loop passes)
    prof, act = b.profile_step()
    dens_gbs = 28.0 * act / (prof.density_ms_total / 1e3) / 1e9
    pf_gbs = 84.0 * act / (prof.pforce_ms_total / 1e3) / 1e9
    try:
        peak, peak_src = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    if prof.pforce_ms_total >= prof.density_ms_total:
        kname, achieved, kms = "k_pcisph_pressure_force<batched>", pf_gbs, prof.pforce_ms_total
    else:
        kname, achieved, kms = "k_pcisph_density<batched>", dens_gbs, prof.density_ms_total

    # end to end: the same steps from the same checkpoint, the host carrying
    # the trajectory. Per step: upload all scenes' positions and velocities
    # from pinned host memory, step, read them back into the same host
    # arrays and wait; the next step's input is that readback.
    b.restore(0)
    b.reset_counters()
    hp = torch.empty((npart, 4), dtype=torch.float32, pin_memory=True)
    hv = torch.empty((npart, 4), dtype=torch.float32, pin_memory=True)
    L = upf.lib()
    fp = C.POINTER(C.c_float)
    upf.check(L.upf_batch_download_state(b.handle, C.cast(hp.data_ptr(), fp), C.cast(hv.data_ptr(), fp)), "dl")

    def e2e_steps():
        for _ in range(args.steps):
            upf.check(L.upf_batch_upload_state_async(b.handle, C.cast(hp.data_ptr(), fp), C.cast(hv.data_ptr(), fp)),
                      "upf_batch_upload_state_async")
            b.step(1)
            upf.check(L.upf_batch_download_state_async(b.handle, C.cast(hp.data_ptr(), fp),
                                                       C.cast(hv.data_ptr(), fp)), "upf_batch_download_state_async")
            upf.check(L.upf_batch_wait_frames(b.handle), "upf_batch_wait_frames")

    e2e_ms = timed(e2e_steps)
    e2e_same = [st.total_iterations for st in b.stats()] == [st.total_iterations for st in stats]
    b.close()

    # baseline: the same scenes as single-scene systems, one after another
    systems = []
    for sc in scs:
        p = upf.derive_params(sc.params)
        s = upf.ParticleSystem(p, capacity=sc.n, device=local_rank, derive=False)
        s.set_stream(stream.cuda_stream)
        s.set_particles(sc.pos, sc.vel, sc.type)
        systems.append(s)
    for s in systems:
        s.step(args.warmup)
    torch.cuda.synchronize()

    def seq():
        for _ in range(args.steps):
            for s in systems:
                s.step(1)

    seq_ms = timed(seq)
    for s in systems:
        s.synchronize()
        s.close()
    seq_value = ns * args.steps * world / (seq_ms / 1e3)
    if rank != 0:
        return
    radix = lambda bits: 3 * ((bits + 7) // 8)  # noqa: E731
    per_step = radix(31) + 1 + radix(8) + 1 + 1 + 1 + 1 + 1 + 1 + 1  # sort, digits, reorder, cells, inits, nlist, ext, integrate
    max_it = max(st.total_iterations for st in stats)
    out = {
        "metric": "batched scene-steps/s (256 PCISPH scenes, 2k-65k particles) vs sequential single-scene steps",
        "value": value, "unit": "scene-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": batch_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched_pcisph_256_scenes", "scenes": ns, "particles": npart,
                   "mean_iterations_per_scene": float(np.mean(its)), "max_iterations_per_scene": float(np.max(its)),
                   "max_density_error_percent_last_step": float(np.max(errs)),
                   "particle_steps_per_s": npart * args.steps * world / (batch_ms / 1e3),
                   "parallelism": "replicas" if world > 1 else "single", "launch_config": tuned,
                   "l2": "inputs larger than L2 (neighbour lists %.0f MB)" % (npart * 128 * 6 / 1e6)},
        "sequential_single_scene": {"value": seq_value, "unit": "scene-steps/s", "ms_per_step": seq_ms / args.steps,
                                    "speedup_of_batched": value / seq_value},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": None, "kernel_ms_per_step": kms,
                     "loop_particle_passes": act},
        "phases_ms": {"sort": prof.sort_ms, "neighbors": prof.neighbors_ms, "forces": prof.forces_ms,
                      "loop": prof.loop_ms, "integrate": prof.integrate_ms, "iterations": prof.iterations},
        "e2e": {"value": ns * args.steps * world / (e2e_ms / 1e3), "unit": "scene-steps/s",
                "h2d_bytes_per_step": npart * 32, "d2h_bytes_per_step": npart * 32, "ms_per_step": e2e_ms / args.steps,
                "input_of_each_step": "the previous step's readback (positions and velocities of every scene)",
                "same_steps_as_value": bool(e2e_same)},
        "gpu_launches": args.steps * per_step + 3 * max_it,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = batch_cpu_baseline(scs, args.cpu_seconds)
    print(json.dumps(out), flush=True)


def run_adjoint(args, rank, world, local_rank):
    """--scene c5: the differentiation form. 65,536 particles (32x32x64
    lattice, initial velocities N(0, 0.1) m/s), 200 steps at dt = 1e-3, 3
    predict-correct iterations per step, checkpoints every 20 steps; loss =
    |x_com(T) - target|^2 + 1e-6 mean (rho - rho0)^2. Reports the forward and
    backward device times and their ratio; the value is the backward's
    particle-steps per second."""
    import torch
    import unifiedparticleframeworkcuda_b200 as upf
    from unifiedparticleframeworkcuda_b200 import build as upfbuild
    from unifiedparticleframeworkcuda_b200 import scenes

    if rank == 0:
        upfbuild.build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sc = scenes.adjoint_scene(32, 32, 64, seed=77 + rank)
    p = upf.derive_params(sc.params)
    T = args.adjoint_steps
    tgt = sc.pos[:, :3].astype(np.float64).mean(0) + np.array([0.1, 0.0, 0.0])
    stream = torch.cuda.Stream(device=dev)
    a = upf.Adjoint(p, sc.pos, sc.vel, T, checkpoint_interval=20, loop_iterations=3, target=tgt, derive=False,
                    device=local_rank)
    a.set_stream(stream.cuda_stream)
    for _ in range(max(args.warmup, 1)):
        a.forward()
        a.backward()
    fwd, bwd = [], []
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            loss = a.forward()
            g, gm = a.backward()
            f, b = a.times()
            fwd.append(f)
            bwd.append(b)
    f_ms, b_ms = replicas.max_over_ranks(float(np.median(fwd)), float(np.median(bwd)))
    # end to end: the calls a gradient-descent loop on the initial velocities
    # makes, timed on the library stream: each trajectory uploads its initial
    # velocities from host memory (upf_adjoint_forward), runs forward and
    # backward, and reads the gradient back to the host
    # (upf_adjoint_backward); the host then takes a small descent step
    v0 = np.array(sc.vel, np.float32, copy=True)
    e2e_ms = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        a.forward(v0)
        ge, _ = a.backward()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        v0[:, :3] -= 1e-2 * ge
    e2e_med = replicas.max_over_ranks(float(np.median(e2e_ms)))[0]
    a.close()
    if rank != 0:
        return
    n = sc.n
    out = {
        "metric": "adjoint (backward) particle-steps/s, 65,536-particle PCISPH trajectory of 200 steps; bwd/fwd ratio",
        "value": n * T * world / (b_ms / 1e3), "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": b_ms / T, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "adjoint_pcisph_65536x200", "particles": n, "trajectory_steps": T,
                   "checkpoint_interval": 20, "loop_iterations": 3, "density_smoothing": 1e-2,
                   "forward_ms": f_ms, "backward_ms": b_ms, "bwd_fwd_ratio": b_ms / f_ms, "loss": loss,
                   "grad_norm": float(np.linalg.norm(g)), "dloss_dviscosity": gm,
                   "timing": "median over the timed forward/backward pairs, CUDA events on the library stream",
                   "l2": "per-interval lists and intermediates ~0.9 GB (larger than L2)"},
        "e2e": {"value": n * T * world / (e2e_med / 1e3), "unit": "particle-steps/s (forward + backward)",
                "h2d_bytes_per_step": n * 16 // T, "d2h_bytes_per_step": n * 16 // T,
                "ms_per_trajectory": e2e_med,
                "calls": "upf_adjoint_forward with the initial velocities from host memory, upf_adjoint_backward "
                         "with the gradient read back; median over the timed trajectories"},
        "gpu_launches": None,
        "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)


def run_io(args, rank, world, local_rank):
    """State files of the 1M dam after one step: a "step" reads the state
    back from the device and writes and re-reads it in each format, the
    reference's liquid dump (UnifiedIO::SaveLiquidParticleInfoFull), the
    PCISPH-format text file (ReadInFluidParticlesPCISPH's input) and the
    binary snapshot file, in a temporary directory on the box's local disk.
    The value is particle records per second through the liquid dump
    (readback included); the reference writer, compiled from its sources
    (oracle/_ref), formats a bounded sample of the same records for the
    baseline."""
    import tempfile

    import torch
    import unifiedparticleframeworkcuda_b200 as upf
    from unifiedparticleframeworkcuda_b200 import build as upfbuild
    from unifiedparticleframeworkcuda_b200 import particle_files as pf

    if rank == 0:
        upfbuild.build()
    torch.cuda.set_device(local_rank)
    sc = scene_for(argparse.Namespace(scene="c2"))
    p = upf.derive_params(sc.params)
    s = upf.ParticleSystem(p, capacity=sc.n, device=local_rank, derive=False)
    s.set_particles(sc.pos, sc.vel, sc.type)
    s.step(1)
    s.synchronize()
    nd = dynamic_count(sc)
    phases = {"readback": 0.0, "liquid_dump": 0.0, "pcisph_text_write": 0.0, "pcisph_text_read": 0.0,
              "snapshot_write": 0.0, "snapshot_read": 0.0}
    sizes = {}
    with tempfile.TemporaryDirectory(dir=os.environ.get("UPF_IO_DIR")) as d:
        def one(timed):
            t = {}
            t0 = time.perf_counter()
            st = s.particles()
            t["readback"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            pf.save_liquid_info_full(os.path.join(d, "liquid.txt"), st["pos"], st["type"])
            t["liquid_dump"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            pf.save_fluid_particles_pcisph(os.path.join(d, "fluid.txt"), st["pos"], st["vel"], st["type"],
                                           st["pressure"], st["density"])
            t["pcisph_text_write"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            back = pf.read_fluid_particles_pcisph(os.path.join(d, "fluid.txt"))
            t["pcisph_text_read"] = time.perf_counter() - t0
            assert back["type"].size == nd
            t0 = time.perf_counter()
            s.write_state_file(os.path.join(d, "state.upf"))
            t["snapshot_write"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            s.read_state_file(os.path.join(d, "state.upf"))
            t["snapshot_read"] = time.perf_counter() - t0
            if timed:
                for k, v in t.items():
                    phases[k] += v
            return st

        for _ in range(args.warmup):
            st = one(False)
        for _ in range(args.steps):
            st = one(True)
        for name in ("liquid.txt", "fluid.txt", "state.upf"):
            sizes[name] = os.path.getsize(os.path.join(d, name))
        base = None
        if not args.no_cpu_baseline:
            base = io_reference_baseline(st, d)
    s.close()
    if rank != 0:
        return
    per = {k: v / args.steps for k, v in phases.items()}
    dump_s = per["readback"] + per["liquid_dump"]
    value = nd / dump_s
    mbs = {"liquid_dump_MBps": sizes["liquid.txt"] / per["liquid_dump"] / 1e6,
           "pcisph_text_write_MBps": sizes["fluid.txt"] / per["pcisph_text_write"] / 1e6,
           "pcisph_text_read_MBps": sizes["fluid.txt"] / per["pcisph_text_read"] / 1e6,
           "snapshot_write_MBps": sizes["state.upf"] / per["snapshot_write"] / 1e6,
           "snapshot_read_MBps": sizes["state.upf"] / per["snapshot_read"] / 1e6}
    out = {"metric": "particle records/s, reference-format liquid dump of the 1M dam state (readback included)",
           "value": value, "unit": "records/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": sum(per.values()) * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "pcisph_dam_break_1M state files", "dynamic_particles": nd,
                      "file_bytes": sizes, "host_threads": os.cpu_count()},
           "phases_ms": {k: v * 1e3 for k, v in per.items()}, "throughput": mbs,
           "e2e": {"value": value, "unit": "records/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": nd * (16 + 16 + 4 + 4 + 4 + 4)},
           "gpu_launches": None, "note": "host-side file formatting and parsing; the device part is the readback"}
    if base:
        out["cpu_baseline"] = base
    print(json.dumps(out))


MESH_METRIC = "lattice point-face tests/s, filling a 5120-face closed mesh (ObjectLoader::LoadParticles)"


def mesh_workload():
    """A 0.1 m sphere of 5,120 faces (about the reference's largest model,
    banana.obj, 5,592 faces) centred on the origin, at 0.002 m spacing: a
    101^3 lattice."""
    from unifiedparticleframeworkcuda_b200 import scenes
    return scenes.mesh_icosphere(0.1, 4), 0.002


def run_mesh(args, rank, world, local_rank):
    """Mesh filling on the GPU (upf_mesh_particles): each step is one call,
    host face set-up, copies, the inside tests of every lattice point against
    every face, compaction and the particles' readback included, timed by
    the host clock around the synchronous call."""
    import unifiedparticleframeworkcuda_b200 as upf
    from unifiedparticleframeworkcuda_b200 import build as upfbuild
    if rank == 0:
        upfbuild.build()
    tri, spacing = mesh_workload()
    ext = tri.reshape(-1, 3)
    lo = np.minimum(ext.min(0), 0.0)
    hi = np.maximum(ext.max(0), 0.0)
    pts = int(np.prod(np.floor((hi - lo) / spacing) + 1))
    for _ in range(args.warmup):
        out = upf.mesh_particles(tri, spacing, device=local_rank)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = upf.mesh_particles(tri, spacing, device=local_rank)
    dt = (time.perf_counter() - t0) / args.steps
    job = replicas.max_over_ranks(dt)[0]
    if rank != 0:
        return
    tests = pts * len(tri)
    line = {"metric": MESH_METRIC, "value": tests * world / job, "unit": "point-face tests/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": job * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "icosphere_5120_faces_2mm", "faces": len(tri), "lattice_points": pts,
                       "particles": len(out)},
            "e2e": {"value": tests * world / job, "unit": "point-face tests/s",
                    "h2d_bytes_per_step": len(tri) * 72, "d2h_bytes_per_step": len(out) * 16},
            "gpu_launches": args.steps * (4 if len(out) else 3)}
    if world == 1 and not args.no_cpu_baseline:
        cb = mesh_reference_sample(tri)
        if cb:
            line["cpu_baseline"] = cb
    print(json.dumps(line), flush=True)


def mesh_reference_sample(tri, spacing=0.006):
    """The reference's ObjectLoader::LoadParticles (compiled from its sources
    into oracle/_ref) on the same mesh at a coarser spacing (a bounded
    sample, about 43k lattice points), one thread."""
    try:
        from oracle import pyoracle
        if not pyoracle.ref_available():
            return None
    except Exception:  # the pin library is not built
        return None
    from unifiedparticleframeworkcuda_b200 import scenes
    ext = tri.reshape(-1, 3)
    pts = int(np.prod(np.floor((np.maximum(ext.max(0), 0) - np.minimum(ext.min(0), 0)) / spacing) + 1))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "mesh.obj")
        scenes.write_obj(path, tri)
        t0 = time.perf_counter()
        pyoracle.ref_obj_particles(path, (1.0, 1.0, 1.0), spacing)
        dt = time.perf_counter() - t0
    return {"value": pts * len(tri) / dt, "unit": "point-face tests/s", "cores": 1, "kind": "reference",
            "sample": "the same mesh at %g m spacing (%d lattice points)" % (spacing, pts)}


def run_io_reference(args):
    """--impl reference --scene io: the reference's SaveLiquidParticleInfoFull
    (compiled from src/cpu/UnifiedIO.cpp into oracle/_ref) on the 1M dam's
    particles, one record stream; each step one full dump."""
    from oracle import pyoracle
    base = {"impl": "reference", "metric": "particle records/s, reference-format liquid dump of the 1M dam state "
                                           "(readback included)", "unit": "records/s"}
    if not pyoracle.ref_available():
        print(json.dumps(dict(base, unavailable="oracle/_ref/libupfref.so (the compiled reference writer) is not "
                                                "built")), flush=True)
        return
    sc = scene_for(argparse.Namespace(scene="c2"))
    dyn = sc.type != 6
    pos = np.ascontiguousarray(sc.pos[dyn], np.float32)
    if pos.shape[1] == 3:
        pos = np.ascontiguousarray(np.concatenate([pos, np.zeros((len(pos), 1), np.float32)], axis=1))
    typ = np.ascontiguousarray(sc.type[dyn], np.int32)
    nl = int(np.count_nonzero(typ == 2))
    with tempfile.TemporaryDirectory(dir=os.environ.get("UPF_IO_DIR")) as d:
        for _ in range(args.warmup):
            pyoracle.ref_io_write("liquid", d, pos, typ, nl)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pyoracle.ref_io_write("liquid", d, pos, typ, nl)
        dt = time.perf_counter() - t0
    v = len(typ) * args.steps / dt
    print(json.dumps(dict(base, value=v, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                          ms_per_step=1e3 * dt / args.steps, higher_is_better=True, scaling="weak",
                          vs_baseline=None, dtype="f32", data="synthetic",
                          config={"workload": "pcisph_dam_break_1M state files", "dynamic_particles": len(typ)},
                          cpu_baseline={"value": v, "unit": "records/s", "cores": 1, "kind": "reference",
                                        "sample": "SaveLiquidParticleInfoFull on all %d dynamic particles"
                                                  % len(typ)},
                          e2e={"value": v, "unit": "records/s", "h2d_bytes_per_step": 0,
                               "d2h_bytes_per_step": 0})), flush=True)


def io_reference_baseline(st, d, records=200_000):
    """The reference's SaveLiquidParticleInfoFull and ReadInFluidParticlesPCISPH
    (compiled from src/cpu/UnifiedIO.cpp into oracle/_ref) on the first
    `records` particles of the same state, one thread."""
    try:
        from oracle import pyoracle
        if not pyoracle.ref_available():
            return None
    except Exception:  # the pin library is not built
        return None
    pos = np.ascontiguousarray(st["pos"][:records])
    typ = np.ascontiguousarray(st["type"][:records])
    nl = int(np.count_nonzero(typ == 2))
    work = os.path.join(d, "ref")
    os.makedirs(work, exist_ok=True)
    t0 = time.perf_counter()
    pyoracle.ref_io_write("liquid", work, pos, typ, nl)
    t_dump = time.perf_counter() - t0
    return {"value": records / t_dump, "unit": "records/s", "cores": 1, "kind": "reference",
            "sample": "SaveLiquidParticleInfoFull on the first %d particles of the same state" % records}


# pieces of the per-step host round trip in the e2e line (upf_exchange_frame_async)
E2E_CHUNKS = 4


def parse_shape(text):
    """'nlist,external,density_threads,density_rows,pforce_threads,pforce_rows[,density_mode,pforce_mode
    [,nlist_mode]]'"""
    from unifiedparticleframeworkcuda_b200 import UpfLaunchConfig
    v = [int(t) for t in text.split(",")]
    if len(v) not in (6, 8, 9):
        raise SystemExit("--shape needs six, eight or nine integers")
    v += [0, 0, 0][: 9 - len(v)]
    c = UpfLaunchConfig()
    (c.nlist_threads, c.external_threads, c.density_threads, c.density_rows, c.pforce_threads,
     c.pforce_rows, c.density_mode, c.pforce_mode, c.nlist_mode) = v
    return c


def run_ours(args, rank, world, local_rank):
    import torch
    import unifiedparticleframeworkcuda_b200 as upf
    from unifiedparticleframeworkcuda_b200 import build as upfbuild

    if rank == 0:
        upfbuild.build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sc = scene_for(args)
    p = upf.derive_params(sc.params)
    if args.block_size:
        p.block_size = args.block_size
    method = "pcisph" if p.method == upf.METHOD_PCISPH else "wcsph"
    stream = torch.cuda.Stream(device=dev)
    s = upf.ParticleSystem(p, capacity=sc.n, device=local_rank, derive=False)
    s.set_stream(stream.cuda_stream)
    s.set_particles(sc.pos, sc.vel, sc.type)
    if sc.num_bodies:
        s.set_rigid_bodies(sc.body, sc.num_bodies)
    nf, nb = sc.n_fluid, sc.n_boundary
    nd = dynamic_count(sc)

    # the timed steps start from the state after the settle steps (the
    # dam's collapse runs its loop into the 50-iteration cap above 1% density
    # error); the reference arm times the same state
    settle = settle_steps(args)
    if settle:
        s.step(settle)
        s.synchronize()

    # warm-up, then the launch-shape autotuner on the warmed state (untimed;
    # it leaves the state unchanged)
    s.step(args.warmup)
    s.synchronize()
    if args.shape:
        s.set_launch_config(parse_shape(args.shape))
        tuned = s.launch_config().as_dict()
    else:
        tuned = s.autotune(3).as_dict() if not args.no_autotune else s.launch_config().as_dict()
    s.reset_counters()
    # the end-to-end run below replays the same steps from this state
    s.checkpoint(0)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed steps' launches
        start.record(stream)
        s.step(args.steps)
        end.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        barrier()
    elapsed_ms = start.elapsed_time(end)
    s.synchronize()
    stats = s.stats()
    max_ms = replicas.max_over_ranks(elapsed_ms)[0]
    total_iters = stats.total_iterations if method == "pcisph" else 0
    mean_k = total_iters / max(stats.total_steps, 1)
    value = nd * args.steps * world / (max_ms / 1e3)

    # per-phase timings (one profiled step through the phase entry points)
    prof = [s.profile_step() for _ in range(3)]
    pr = prof[-1]
    # dominant kernel: the loop's predicted-density or pressure-force pass
    dens_ms = pr.density_ms_total / max(pr.iterations, 1)
    pf_ms = pr.pforce_ms_total / max(pr.iterations, 1)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    if method == "pcisph":
        # algorithmic bytes per liquid particle: density pass reads predicted
        # position 16 + pressure 4, writes pressure 4 + density 4 = 28;
        # pressure-force pass reads position 16, pressure 4, velocity 16,
        # force 16, writes pressure force 16 + next prediction 16 = 84
        if pf_ms >= dens_ms:
            kname, kms, kbytes = "k_pcisph_pressure_force", pf_ms, 84 * nf
        else:
            kname, kms, kbytes = "k_pcisph_density", dens_ms, 28 * nf
    else:
        kname, kms, kbytes = "k_wcsph_force_integrate", pr.integrate_ms, (16 + 16 + 4 + 4 + 16 + 16 + 4) * nf
    achieved = kbytes / (kms / 1e3) / 1e9
    step_bytes = algorithmic_bytes(nf, nb, args.steps, total_iters, method)
    # DRAM bytes per fluid particle per launch, measured by ncu captures of
    # the same kernels on the 262k-fluid dam (read + write, one launch) and
    # scaled here by the fluid count (the list length per particle does not
    # depend on the scene size); not measured in this run. Keyed by the list
    # mode the tuned shape reads: staged neighbourhoods (mode 2) stream
    # 16-bit union positions in place of 32-bit list entries
    staged = (tuned.get("density_mode" if kname == "k_pcisph_density" else "pforce_mode") == 2)
    traffic_per_particle = {("k_pcisph_density", False): 157.9, ("k_pcisph_density", True): 110.7,
                            ("k_pcisph_pressure_force", False): 361.2, ("k_pcisph_pressure_force", True): 280.8}
    traffic = traffic_per_particle[(kname, staged)] * nf if (kname, staged) in traffic_per_particle else None
    traffic_source = ("ncu dram__bytes_read+write per fluid particle on the 262k-fluid dam, scaled to %d fluid "
                      "particles" % nf) if traffic is not None else None

    # end to end through the C ABI with host buffers, over the same steps as
    # the timed region (restored from the checkpoint): every step uploads its
    # input positions and velocities from pinned host memory, steps, and
    # reads its result back into pinned host memory; the next step's input
    # is that readback, so the host carries the trajectory from frame to
    # frame and the steps are the timed region's steps
    e2e = None
    if not args.no_e2e:
        s.restore(0)
        n = s.n_dynamic
        hpos = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
        hvel = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
        hden = torch.empty((n,), dtype=torch.float32, pin_memory=True)
        hpre = torch.empty((n,), dtype=torch.float32, pin_memory=True)
        htyp = torch.empty((n,), dtype=torch.int32, pin_memory=True)
        hid = torch.empty((n,), dtype=torch.int32, pin_memory=True)
        import ctypes as C
        L = upf.lib()
        fp = C.POINTER(C.c_float)
        cnt = C.c_uint32()

        # upf_*_async run the copies on the library's copy streams; the
        # host waits for each readback before it uploads it as the next
        # step's input, so copies and steps alternate
        def readback():
            upf.check(L.upf_get_particles_async(s.handle, C.cast(hpos.data_ptr(), fp), C.cast(hvel.data_ptr(), fp),
                                                C.cast(hden.data_ptr(), fp), C.cast(hpre.data_ptr(), fp),
                                                C.cast(htyp.data_ptr(), C.POINTER(C.c_int32)),
                                                C.cast(hid.data_ptr(), C.POINTER(C.c_uint32)), C.byref(cnt)),
                      "upf_get_particles_async")

        readback()  # the first step's input: the state at the checkpoint
        upf.check(L.upf_wait_frames(s.handle), "upf_wait_frames")
        s.reset_counters()
        k_e2e = args.steps
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # each step: its input uploaded from the host arrays, the step, its
        # result read back into the host arrays and waited for. After a step
        # the readback and the next step's upload are one host round trip
        # (upf_exchange_frame_async): the upload of each piece of the
        # positions and velocities starts once that piece has reached host
        # memory, so the two copy directions overlap; the bytes uploaded are
        # those read back. The frame's other fields (density, pressure, type,
        # id) come back after its positions and velocities, while the next
        # step runs; the host waits for each whole frame before it queues
        # the next frame's copies, and for the last one before the clock
        # stops.
        upf.check(L.upf_upload_state_async(s.handle, C.cast(hpos.data_ptr(), fp), C.cast(hvel.data_ptr(), fp), n),
                  "upf_upload_state_async")
        for k in range(k_e2e):
            s.step(1)
            if k > 0:
                upf.check(L.upf_wait_frames(s.handle), "upf_wait_frames")  # frame k - 1 is on the host
            if k + 1 < k_e2e:
                upf.check(L.upf_exchange_frame_async(
                    s.handle, C.cast(hpos.data_ptr(), fp), C.cast(hvel.data_ptr(), fp), C.cast(hden.data_ptr(), fp),
                    C.cast(hpre.data_ptr(), fp), C.cast(htyp.data_ptr(), C.POINTER(C.c_int32)),
                    C.cast(hid.data_ptr(), C.POINTER(C.c_uint32)), args.e2e_chunks, C.byref(cnt)),
                    "upf_exchange_frame_async")
            else:
                readback()
        upf.check(L.upf_wait_frames(s.handle), "upf_wait_frames")
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = replicas.max_over_ranks(e0.elapsed_time(e1))[0]
        st_e2e = s.stats()
        e2e = {"value": nd * k_e2e * world / (e2e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": n * (16 + 16 + 4 + 4 + 4 + 4),
               "steps": k_e2e, "ms_per_step": e2e_ms / k_e2e,
               "input_of_each_step": "the previous step's readback (host round trip every step; readback and "
                                     "upload overlapped in %d pieces; the fields that are not the next input "
                                     "read back during the next step)" % args.e2e_chunks,
               "same_steps_as_value": bool(st_e2e.total_iterations == total_iters
                                           and st_e2e.total_steps == stats.total_steps)}

    if rank != 0:
        s.close()
        return
    launches_base = 1 + 1 + 1 + 3 * RADIX_PASSES + 1 + 1  # step init, nlist, forces, sort, reorder, cells
    if method == "pcisph":
        rigid = (1 + 2 + 1) if sc.num_bodies else 0  # slots, reduce + integrate, sync
        staged = 1 if 2 in (tuned.get("density_mode"), tuned.get("pforce_mode")) else 0  # k_stage_lists
        gpu_launches = args.steps * (launches_base + 2 + rigid + staged) + 3 * total_iters
    else:
        gpu_launches = args.steps * (launches_base + 1)
    out = {
        "metric": metric_for(args), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args), "fluid_particles": nf, "boundary_particles": nb,
                   "dynamic_particles": nd, "rigid_bodies": int(sc.num_bodies),
                   "h": float(p.support_radius), "dt": float(p.dt),
                   **({"dt_note": C1_NOTE} if args.scene == "c1" else {}), "block_size": int(p.block_size),
                   "settle_steps": settle, "mean_iterations": mean_k,
                   "steps_at_max_loops": stats.steps_at_max_loops,
                   "max_step_density_error_percent": float(stats.max_step_density_error_percent),
                   "density_criterion_met_every_step": bool(method == "pcisph" and stats.steps_at_max_loops == 0
                                                            and stats.max_step_density_error_percent < p.max_density_error),
                   "last_density_error_percent": float(stats.density_error_percent),
                   "parallelism": "replicas" if world > 1 else "single",
                   "launch_config": tuned,
                   "l2": "inputs larger than L2 (neighbour lists %.0f MB)" % (sc.n * p.max_neighbors * 4 / 1e6)},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                     "traffic_source": traffic_source,
                     "kernel_ms": kms, "algorithmic_bytes_per_launch": kbytes,
                     "step_achieved_gbs": step_bytes / (max_ms / 1e3) / 1e9 / world * world,
                     "step_frac": step_bytes / (max_ms / 1e3) / 1e9 / peak},
        "phases_ms": {"sort": pr.sort_ms, "neighbors": pr.neighbors_ms, "forces": pr.forces_ms,
                      "loop": pr.loop_ms, "integrate": pr.integrate_ms, "iterations": pr.iterations,
                      "density_per_launch": dens_ms, "pforce_per_launch": pf_ms},
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        dam = args.scene in ("c2", "c2-small")
        if dam:
            s.restore(0)  # the state at the start of the timed steps
        out["cpu_baseline"] = cpu_baseline(args, seconds=args.cpu_seconds, system=s if dam else None)
        out["config"]["fp64_err"] = fp64_error(s, sc, os.cpu_count() or 1)
    print(json.dumps(out), flush=True)
    s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scene", default="c2", choices=["c2", "c2-small", "c1", "c3", "c4", "c5", "io", "mesh"])
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--block-size", type=int, default=0)
    ap.add_argument("--settle", type=int, default=-1,
                    help="steps from rest before the warm-up (default: the workload's settle count, after which "
                         "the dam's loop meets the 1%% criterion; 0 = time from rest); both arms time the state "
                         "after them")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-chunks", type=int, default=E2E_CHUNKS,
                    help="pieces of each e2e host round trip (1..16)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--shape", default="", help="fixed launch shapes instead of the autotuner: "
                                                "nlist,external,density_threads,density_rows,pforce_threads,pforce_rows"
                                                "[,density_mode,pforce_mode[,nlist_mode]]")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=60.0,
                    help="bound on the reference arm's timed steps on the host cores (at least 3 run)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    try:
        if args.scene == "c4":
            run_batch(args, rank, world, local_rank)
        elif args.scene == "io":
            run_io(args, rank, world, local_rank)
        elif args.scene == "mesh":
            run_mesh(args, rank, world, local_rank)
        elif args.scene == "c5":
            run_adjoint(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
