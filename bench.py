"""Throughput of the batched soft-body step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the uneven population -- 512 voxel robots with side
uniform in 3..8 cells (64 to 729 masses, up to 7,448 springs each), cell
materials iid {air .3, bone .175, tissue .175, muscle_a .175, muscle_b .175},
seeded synthetic robots -- stepped with the reference's step semantics at
dt = 1e-4 for 1 s of simulated time (10,000 steps, the reference's float
clock).  One bench step = one such evaluation of the whole population.

Metric: spring-updates/s = (non-air springs of all robots) x (steps) /
seconds.  `value` is device-timed (CUDA events on the context's stream) with
the population resident in HBM; `e2e` is wall-timed through the C ABI with
host buffers: upload of the population from pinned memory (mb_set_elements),
mb_simulate, and the read-back of positions, velocities, stresses and centres
of mass.  With N GPUs (torchrun) every rank simulates its own population of
the same shape (weak scaling) and timings are the max over ranks.

--impl reference: the reference's step on this box.  Its `value` is the CPU
restatement of the reference step (oracle, OpenMP over all host cores) on a
bounded sample of the same workload; the line also carries the reference's
own CUDA simulator (built from its sources into oracle/_ref) timed on the
GPU on the same population, padded to equal mass counts as it requires.
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

WORKLOADS = {
    # name: (population, duration s, dt, track stresses)
    "uneven": ("uneven", 1.0, 1e-4, False),
    "small": ("small", 1.0, 1e-4, False),
    "streamed": ("streamed", 0.1, 1e-4, True),
}

# Algorithmic bytes per spring-update.
#   Shared memory (the binding resource of the resident step kernel, which
#   keeps every robot on chip for a whole launch): 24 B for the two endpoint
#   positions (2 x 3 floats) + 12 B for the correction the spring stores
#   (3 floats) + 24 B for the two reads of that correction when its ends
#   gather it (2 x 3 floats) = 60 B.
#   HBM, for a step that keeps nothing on chip (the reference's design):
#   9 B topology (2 x u16 pair, u8 material, f32 mean length) + 8 B stress
#   read+write when tracking + per-mass state (pos and vel, 3 floats each,
#   read and write: 48 B) x masses/springs.
SMEM_B = 60.0
SMEM_NOMINAL_B_PER_CLK = 128.0  # shared-memory bandwidth of an SM (32 banks x 4 B per clock)
HBM_TOPO_B, HBM_STRESS_B, HBM_MASS_B = 9.0, 8.0, 48.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


class Pinned:
    """Keeps pinned host copies of a batch's arrays alive."""

    def __init__(self, batch):
        import torch
        self._t = []
        self.arrays = {}
        for name in ("mass_offsets", "pos", "vel", "mass_material", "spring_offsets", "pairs",
                     "spring_material", "lbar"):
            a = getattr(batch, name)
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            v = t.numpy().view(a.dtype).reshape(a.shape)
            v[...] = a
            self._t.append(t)
            self.arrays[name] = v

    def batch(self, like):
        from mercury_b200.element import Batch
        return Batch(**self.arrays)

    def empty(self, shape, dtype):
        import torch
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        t = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        self._t.append(t)
        return t.numpy().view(dtype).reshape(shape)


def cpu_baseline(batch, dt, track, seconds_target=15.0):
    """Oracle (C restatement, OpenMP over robots) on a bounded sample: all
    robots, a number of steps sized to ~seconds_target of work."""
    import mercury_b200 as mb
    from oracle import core
    threads = os.cpu_count() or 1
    table = mb.material_table()
    active = batch.active_springs()
    # calibrate on 20 steps
    p, v = batch.pos.copy(), batch.vel.copy()
    s = np.zeros(batch.n_springs, np.float32)
    t0 = time.perf_counter()
    core.xpbd_run(batch, p, v, s, table, dt, 0.0, 20, track, threads)
    rate = active * 20 / max(time.perf_counter() - t0, 1e-9)
    steps = int(max(20, min(5000, seconds_target * rate / active)))
    p, v = batch.pos.copy(), batch.vel.copy()
    s = np.zeros(batch.n_springs, np.float32)
    t0 = time.perf_counter()
    core.xpbd_run(batch, p, v, s, table, dt, 0.0, steps, track, threads)
    el = time.perf_counter() - t0
    return {"value": active * steps / el, "unit": "spring-updates/s", "cores": threads, "kind": "port",
            "sample": f"all {batch.n_robots} robots, first {steps} steps of the workload ({el:.1f} s)"}


def run_ours(args, rank, local_rank, world):
    import torch

    import mercury_b200 as mb
    from mercury_b200 import dist, robots

    pop, duration, dt, track = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    batch = robots.population_batch(pop, seed_base=dist.seed_base(1000 * {"small": 0, "uneven": 1, "streamed": 4}[pop], rank))
    active = batch.active_springs()
    sim = mb.Simulator(local_rank)
    sim.setTimeStep(dt)
    sim.set_batch(batch)
    tuned = None
    if not args.no_autotune:
        from mercury_b200 import autotune
        tuned = autotune.tune(sim, batch, track=track, steps=300, use_cache=args.autotune_cache)
    steps_per_eval = None

    stream = torch.cuda.ExternalStream(sim.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def one_eval():
        sim.set_state(batch.pos, batch.vel)
        sim.Reset()
        return sim.Simulate(duration, trackStresses=track)

    for _ in range(args.warmup):
        steps_per_eval = one_eval()
    sim.synchronize()
    cfg = sim.launch_config()
    launches_per_eval = -(-steps_per_eval // cfg["chunk"])

    dist.barrier()
    times = []
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed iterations (256 MB > 126 MB L2)
            sim.set_state(batch.pos, batch.vel)
            sim.Reset()
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.Simulate(duration, trackStresses=track)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        torch.cuda.synchronize(dev)
    dist.barrier()
    t_local = float(np.sum(times))
    t_max = dist.max_over_ranks(t_local, dev)
    updates_local = float(active) * steps_per_eval * args.steps
    updates_all = dist.sum_over_ranks(updates_local, dev)
    value = updates_all / t_max
    ms_per_step = 1e3 * t_max / args.steps

    # roofline of the step kernel (per launch): shared-memory bound, against
    # the shared-memory read bandwidth measured on this GPU by the probe kernel
    t_launch = t_local / (args.steps * launches_per_eval)
    upd_launch = float(active) * steps_per_eval / launches_per_eval
    hbm_b = HBM_TOPO_B + (HBM_STRESS_B if track else 0.0) + HBM_MASS_B * batch.n_masses / active
    hbm_peak, hbm_src = peaks()
    clocks = clk.summary()
    smem_peak, smem_clk = smem_peak_gbs(local_rank)
    hbm_ach = hbm_b * upd_launch / t_launch / 1e9
    smem_ach = SMEM_B * upd_launch / t_launch / 1e9

    # plain configuration: one robot per CTA, one step per launch, no graph
    plain = None
    if not args.no_plain:
        psim = mb.Simulator(local_rank)
        psim.setTimeStep(dt)
        psim.set_launch_config(bins=batch.n_robots, chunk=1, use_graph=0)
        psim.set_batch(batch)
        pstream = torch.cuda.ExternalStream(psim.stream, device=dev)
        psim.run_steps(50, track)
        psim.synchronize()
        n_plain = 1000
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(pstream)
        psim.run_steps(n_plain, track)
        e1.record(pstream)
        e1.synchronize()
        tp = dist.max_over_ranks(e0.elapsed_time(e1) / 1e3, dev)
        plain = dist.sum_over_ranks(float(active) * n_plain, dev) / tp
        del psim

    # end to end through the C ABI with host buffers (pinned)
    pinned = Pinned(batch)
    hb = pinned.batch(batch)
    out_pos = pinned.empty((batch.n_masses, 4), np.float32)
    out_vel = pinned.empty((batch.n_masses, 4), np.float32)
    out_st = pinned.empty((batch.n_springs,), np.float32)
    esim = mb.Simulator(local_rank)
    esim.setTimeStep(dt)
    if tuned is not None:  # the launch configuration chosen above, as a user would reuse it
        esim.set_launch_config(**{k: cfg[k] for k in ("threads", "springs_per_thread", "masses_per_thread",
                                                      "bins", "chunk", "use_graph", "streamed")})
    esim.set_batch(hb)
    esim.Simulate(duration, track)  # warm: graph built for this clock
    esim.synchronize()
    e_steps = max(1, min(args.steps, 5))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e_steps):
        esim.set_batch(hb)
        esim.Reset()
        esim.Simulate(duration, trackStresses=track)
        esim.collect_arrays((out_pos, out_vel, out_st))
        esim.CentreOfMass()
    e2e_t = dist.max_over_ranks(time.perf_counter() - t0, dev)
    e2e_launch = esim.launch_config()
    e2e = dist.sum_over_ranks(float(active) * steps_per_eval * e_steps, dev) / e2e_t
    h2d = sum(a.nbytes for a in pinned.arrays.values())
    d2h = out_pos.nbytes + out_vel.nbytes + out_st.nbytes + 12 * batch.n_robots

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(batch, dt, track)

    # single-GPU lines beside the headline: measured at N = 1 only (at N > 1
    # every GPU would repeat them while all are held)
    extra = {} if (args.no_extra or world > 1) else secondary(args, batch, local_rank, dev, hbm_peak)

    line = {
        "metric": "spring-updates/s",
        "value": value,
        "unit": "spring-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "vs_plain": (value / plain) if plain else None,
        "plain": {"value": plain, "unit": "spring-updates/s",
                  "config": "one robot per CTA, one step per launch, no graph, 1,000 steps"} if plain else None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"{args.workload}: {batch.n_robots} voxel robots per GPU, "
                        f"{batch.n_masses} masses, {batch.n_springs} springs ({active} non-air), "
                        f"reference XPBD step, dt={dt}, {duration} s = {steps_per_eval} steps per bench step",
            "robots_per_gpu": batch.n_robots,
            "steps_per_bench_step": steps_per_eval,
            "active_springs_per_gpu": active,
            "launch": cfg,
            "l2": "flushed between timed iterations (256 MB write)",
            "parallelism": f"population sharded over {world} GPU(s), no collective in the step",
        },
        "roofline": {"bound": "smem", "achieved": smem_ach, "peak": smem_peak, "unit": "GB/s",
                     "frac": smem_ach / smem_peak, **_step_traffic(args.workload, cfg, active),
                     "bytes_per_update": SMEM_B,
                     "peak_source": f"measured: shared-memory read probe (mb_measure_smem_bandwidth) on this GPU, "
                                    f"{smem_clk:.1f} B/clk/SM",
                     "kernel": "step_kernel (resident: robots on chip for the whole launch)"},
        "roofline_hbm": {"bound": "hbm", "achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s",
                         "frac": hbm_ach / hbm_peak, "bytes_per_update": hbm_b, "peak_source": hbm_src,
                         "note": "the HBM bytes a step that keeps nothing on chip (the reference's design) "
                                 "must move per spring-update; this kernel moves the state and topology "
                                 "once per launch (traffic)"},
        "kernel_ms_per_launch": 1e3 * t_launch,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "spring-updates/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e_steps, "launch": e2e_launch},
        "gpu_launches": int(2 * launches_per_eval * args.steps),
        "gpu_launches_note": "per chunk of steps: one actuation-table launch and one step launch",
        "clocks": clocks,
        "autotune": ({"candidates": len(tuned.get("candidates", [])), "cached": "candidates" not in tuned,
                      "chosen": tuned["config"]} if tuned else None),
        **extra,
    }
    return line


def _device_rate(sim, active, steps, track, dev):
    import torch
    st = torch.cuda.ExternalStream(sim.stream, device=dev)
    sim.run_steps(min(200, steps), track)
    sim.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.run_steps(steps, track)
    e1.record(st)
    e1.synchronize()
    return active * steps / (e0.elapsed_time(e1) / 1e3)


# DRAM bytes (read + write) of one 1,000-step launch of the step kernel on
# the uneven population in the configurations the tuner picks (ncu,
# dram__bytes_read.sum + dram__bytes_write.sum): the state and topology, read
# once per launch.
STEP_TRAFFIC = {("uneven", 1024, 8, 2, 296, 1000): 24.664e6 + 0.0,
                ("uneven", 1024, 10, 2, 296, 1000): 24.666e6 + 0.0}


def _step_traffic(workload, cfg, active):
    """Measured DRAM bytes per launch, when the bench runs the profiled
    configuration."""
    key = (workload, cfg["threads"], cfg["springs_per_thread"], cfg["masses_per_thread"], cfg["bins"], cfg["chunk"])
    t = STEP_TRAFFIC.get(key)
    if t is None:
        return {"traffic": None}
    return {"traffic": t, "traffic_unit": "DRAM bytes per launch",
            "traffic_source": "ncu capture of the same configuration (dram__bytes_read.sum + dram__bytes_write.sum)"}


def smem_peak_gbs(device):
    """Shared-memory read bandwidth of this GPU (GB/s) and bytes per clock
    per SM, from the library's probe kernel."""
    import ctypes

    from mercury_b200 import _lib
    bps, bpc = ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.LIB.mb_measure_smem_bandwidth(device, ctypes.byref(bps), ctypes.byref(bpc)))
    if bpc.value > 1.05 * SMEM_NOMINAL_B_PER_CLK:
        raise RuntimeError(f"shared-memory probe measured {bpc.value:.1f} B/clk/SM, above the "
                           f"{SMEM_NOMINAL_B_PER_CLK:.0f} B/clk/SM the SM can serve: loads were merged")
    return bps.value / 1e9, bpc.value


def secondary(args, batch, local_rank, dev, hbm_peak):
    """Beside the headline: the force modes (the benchmark configurations'
    physics) on the same robots with 0.1 kg masses, and the robots too large
    for one CTA -- 64 of 10x10x10 cells (1,331 masses, 14,230 springs each)
    and 256 point clouds of 500-2,000 masses in water, stresses tracked --
    on the default path (split over thread-block clusters) and on the
    streamed kernel, with the streaming step's HBM figure."""
    import mercury_b200 as mb
    from mercury_b200 import robots
    from mercury_b200 import simulator as S
    out = {}
    fb = mb.Batch(**{k: getattr(batch, k) for k in ("mass_offsets", "pos", "vel", "mass_material",
                                                    "spring_offsets", "pairs", "spring_material", "lbar")})
    fb.pos = batch.pos.copy()
    fb.pos[:, 3] = 0.1
    for name, mode, env in (("force_land", S.MODE_FORCE_LAND, S.LAND),
                            ("force_water", S.MODE_FORCE_WATER, S.WATER)):
        fs = mb.Simulator(local_rank)
        fs.set_materials(mb.materials.force_table())
        fs.set_mode(mode)
        fs.set_environment(**env)
        fs.setTimeStep(1e-4)
        fs.set_batch(fb)
        rate = _device_rate(fs, fb.active_springs(), 5000, False, dev)
        p, _, _ = fs.collect_arrays()
        out[name] = {"value": rate, "unit": "spring-updates/s", "steps": 5000,
                     "finite": bool(np.isfinite(p).all()), "config": fs.launch_config()}
        del fs
    # water with the face drag: the same robots with their exposed cell faces
    # (two triangles per square), drag on the faces instead of per mass
    els = robots.population("uneven", batch.n_robots, mass=0.1, faces=True)
    wb = mb.pack(els)
    fs = mb.Simulator(local_rank)
    fs.set_materials(mb.materials.force_table())
    fs.set_mode(S.MODE_FORCE_WATER)
    fs.set_environment(**S.WATER_FACES)
    fs.setTimeStep(1e-4)
    fs.set_batch(wb)
    rate = _device_rate(fs, wb.active_springs(), 5000, False, dev)
    p, _, _ = fs.collect_arrays()
    n_faces = int(wb.face_offsets[-1])
    out["force_water_faces"] = {
        "value": rate, "unit": "spring-updates/s", "steps": 5000, "finite": bool(np.isfinite(p).all()),
        "faces": n_faces, "face_updates_per_s": rate * n_faces / wb.active_springs(),
        "workload": f"the headline robots with 0.1 kg masses and {n_faces} surface triangles, water, "
                    f"face drag rho = {S.WATER_FACES['face_drag']:g} (no per-mass drag)",
        "config": fs.launch_config()}
    del fs
    def large(batch, mode, env, workload):
        """Default path (robots split over thread-block clusters) and, for
        comparison, the streamed kernel (never split)."""
        act = batch.active_springs()
        hbm_b = HBM_TOPO_B + HBM_STRESS_B + HBM_MASS_B * batch.n_masses / act
        res = {}
        for key, cfg in (("split", {}), ("streamed", {"cluster": 1})):
            sim = mb.Simulator(local_rank)
            if mode:
                sim.set_materials(mb.materials.force_table())
                sim.set_mode(mode)
                sim.set_environment(**env)
            sim.setTimeStep(1e-4)
            sim.set_launch_config(**cfg)
            sim.set_batch(batch)
            rate = _device_rate(sim, act, 1000, True, dev)
            p, _, _ = sim.collect_arrays()
            res[key] = {"value": rate, "config": sim.launch_config(), "finite": bool(np.isfinite(p).all()),
                        "roofline": {"bound": "hbm", "achieved": rate * hbm_b / 1e9, "peak": hbm_peak,
                                     "unit": "GB/s", "frac": rate * hbm_b / 1e9 / hbm_peak,
                                     "bytes_per_update": hbm_b,
                                     "note": "HBM bytes a streaming step moves per spring-update"}}
            del sim
        return {"value": res["split"]["value"], "unit": "spring-updates/s", "steps": 1000,
                "workload": workload, "config": res["split"]["config"], "finite": res["split"]["finite"],
                "vs_streamed": res["split"]["value"] / res["streamed"]["value"], "streamed_kernel": res["streamed"]}

    sb = robots.population_batch("streamed", 64, seed_base=4000)
    out["streamed"] = large(sb, 0, None,
                            f"64 robots of 10x10x10 cells, {sb.n_masses} masses, {sb.active_springs()} springs, "
                            f"stresses tracked, reference step, dt=1e-4")
    out["long_horizon"] = long_horizon(sb, local_rank, dev, hbm_peak)
    out["force_land_divergence"] = land_divergence(local_rank)
    # point-cloud robots in water (256 robots of 500-2,000 masses, 25 nearest
    # neighbours, stresses tracked): springs built on the device
    nb = mb.pack(robots.nn_population_device(256, mass=0.1, device=local_rank))
    out["nn_water"] = large(nb, S.MODE_FORCE_WATER, S.WATER,
                            f"256 point-cloud robots of 500-2,000 masses, 25 nearest-neighbour springs, "
                            f"{nb.n_masses} masses, {nb.active_springs()} springs, water, stresses tracked, "
                            f"dt=1e-4")
    # the same point clouds with their convex hulls as surfaces and the face
    # drag on (split over clusters, velocities exchanged with positions)
    hb = mb.Batch(**{k: getattr(nb, k) for k in ("mass_offsets", "pos", "vel", "mass_material",
                                                 "spring_offsets", "pairs", "spring_material", "lbar")})
    hulls = [robots.hull_faces(nb.pos[int(nb.mass_offsets[r]):int(nb.mass_offsets[r + 1]), :3])
             for r in range(nb.n_robots)]
    hb.face_offsets = np.concatenate([[0], np.cumsum([len(h) for h in hulls])]).astype(np.int64)
    hb.faces = np.ascontiguousarray(np.concatenate(hulls), np.uint16)
    fs = mb.Simulator(local_rank)
    fs.set_materials(mb.materials.force_table())
    fs.set_mode(S.MODE_FORCE_WATER)
    fs.set_environment(**S.WATER_FACES)
    fs.setTimeStep(1e-4)
    fs.set_batch(hb)
    rate = _device_rate(fs, hb.active_springs(), 1000, True, dev)
    p, _, _ = fs.collect_arrays()
    out["nn_water_faces"] = {
        "value": rate, "unit": "spring-updates/s", "steps": 1000, "finite": bool(np.isfinite(p).all()),
        "faces": int(hb.face_offsets[-1]), "config": fs.launch_config(),
        "workload": "the nn_water robots with their convex hulls as surfaces, face drag rho = 1000 "
                    "(no per-mass drag), stresses tracked"}
    del fs
    out["devo"] = devo_bench(local_rank)
    out["build"] = build_bench(local_rank)
    out["surrogate"] = surrogate_bench(local_rank)
    return out


def long_horizon(sb, local_rank, dev, hbm_peak):
    """The streamed long-horizon configuration as specified: 64 robots of
    10x10x10 cells, stresses tracked, Simulate(10 s) at dt = 1e-4 (99,937
    steps of the float clock), device-timed on the default path (robots split
    over thread-block clusters); with the drift of the FP32 positions from
    the oracle's FP64 transcription over the first 1,000 steps."""
    import torch

    import mercury_b200 as mb
    from oracle import core
    act = sb.active_springs()
    sim = mb.Simulator(local_rank)
    sim.setTimeStep(1e-4)
    sim.set_batch(sb)
    sim.run_steps(1000, True)
    pos, _, _ = sim.collect_arrays()
    pd, vd = sb.pos.astype(np.float64), sb.vel.astype(np.float64)
    sd = np.zeros(sb.n_springs, np.float64)
    core.xpbd_run_f64(sb, pd, vd, sd, core.material_table(), 1e-4, 0.0, 1000, True)
    drift = float(np.abs(pos[:, :3] - pd[:, :3]).max())
    motion = float(np.abs(pd[:, :3] - sb.pos[:, :3]).max())
    sim.set_state(sb.pos, sb.vel)
    sim.Reset()
    st = torch.cuda.ExternalStream(sim.stream, device=dev)
    sim.Simulate(0.01, trackStresses=True)  # warm: graph of the chunk
    sim.set_state(sb.pos, sb.vel)
    sim.Reset()
    sim.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    steps = sim.Simulate(10.0, trackStresses=True)
    e1.record(st)
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    p, _, _ = sim.collect_arrays()
    rate = act * steps / secs
    hbm_b = HBM_TOPO_B + HBM_STRESS_B + HBM_MASS_B * sb.n_masses / act
    return {"value": rate, "unit": "spring-updates/s", "steps": steps, "seconds": secs,
            "simulated_s": 10.0, "finite": bool(np.isfinite(p).all()), "config": sim.launch_config(),
            "roofline": {"bound": "hbm", "achieved": rate * hbm_b / 1e9, "peak": hbm_peak, "unit": "GB/s",
                         "frac": rate * hbm_b / 1e9 / hbm_peak, "bytes_per_update": hbm_b,
                         "note": "HBM bytes a streaming step moves per spring-update (the split kernel keeps "
                                 "each robot on chip over two SMs)"},
            "drift_vs_fp64_first_1000_steps_m": drift, "fp64_motion_first_1000_steps_m": motion,
            "workload": f"64 robots of 10x10x10 cells ({sb.n_masses} masses, {act} springs), stresses tracked, "
                        f"reference step, dt=1e-4, Simulate(10 s)"}


def land_divergence(local_rank):
    """Contact chaos: max |x_fp32 - x_fp64| of the land mode on 32 uneven
    robots (0.1 kg masses), the CUDA step against the oracle's FP64
    transcription of the same law, after 10 ... 3,000 steps."""
    import mercury_b200 as mb
    from mercury_b200 import robots
    from mercury_b200 import simulator as S
    from oracle import core
    keys = ("g", "floor_stiffness", "friction_static", "friction_kinetic", "drag", "damping")
    b = robots.population_batch("uneven", 32, mass=0.1)
    sim = mb.Simulator(local_rank)
    sim.set_materials(mb.materials.force_table())
    sim.set_mode(S.MODE_FORCE_LAND)
    sim.set_environment(**S.LAND)
    sim.setTimeStep(1e-4)
    sim.set_batch(b)
    pd, vd = b.pos.astype(np.float64), b.vel.astype(np.float64)
    done, curve = 0, {}
    for n in (10, 30, 100, 300, 1000, 3000):
        sim.run_steps(n - done, False)
        core.force_run_f64(1, b, pd, vd, mb.materials.force_table(), [S.LAND[k] for k in keys], 1e-4,
                           done * 1e-4, n - done)
        done = n
        pos, _, _ = sim.collect_arrays()
        curve[str(n)] = float(np.abs(pos[:, :3] - pd[:, :3]).max())
    g = np.log(curve["1000"] / curve["30"]) / 970.0
    return {"max_abs_dx_m": curve, "growth_per_step": float(g), "efold_steps": float(1.0 / g),
            "workload": "32 uneven voxel robots, 0.1 kg masses, land (penalty ground, Coulomb friction), dt=1e-4"}


def build_bench(local_rank):
    """Robot construction (optimize/benchmark.cpp "build" mode), robots/s:
    4096 random 6x6x6 voxel genomes built and packed on the device
    (mb_set_voxel_population) against the host builder plus host packing on
    512 of them; the k = 25 nearest-neighbour springs of 256 point-cloud
    robots (the third configuration) on the device (mb_knn_springs) against
    the host builder on 16 of them."""
    import mercury_b200 as mb
    from mercury_b200 import evolve, robots
    from mercury_b200.surrogate import to_cells
    rng = np.random.default_rng(5)
    cells = to_cells(evolve.random_genomes(rng, 4096))
    sim = mb.Simulator(local_rank)
    sim.set_voxel_population(cells, 0.1, 0.1)  # plans the packing once
    t0 = time.perf_counter()
    for _ in range(3):
        sim.set_voxel_population(cells, 0.1, 0.1)
    dev_vox = 3 * 4096 / (time.perf_counter() - t0)
    t0 = time.perf_counter()
    b = mb.pack([robots.voxel_robot(c, 0.1, 0.1) for c in cells[:512]])
    hs = mb.Simulator(local_rank)
    hs.set_batch(b)
    host_vox = 512 / (time.perf_counter() - t0)
    pts, mats = [], []
    for r in range(256):
        g = np.random.default_rng(2000 + r)
        p, m = robots.nn_points(g, int(g.integers(500, 2001)))
        pts.append(p)
        mats.append(m)
    robots.knn_springs(pts[:8], mats[:8])
    t0 = time.perf_counter()
    robots.knn_springs(pts, mats)
    dev_knn = 256 / (time.perf_counter() - t0)
    t0 = time.perf_counter()
    for r in range(16):
        g = np.random.default_rng(2000 + r)
        robots.nn_robot(g, int(g.integers(500, 2001)))
    host_knn = 16 / (time.perf_counter() - t0)
    return {"unit": "robots/s",
            "voxel_6x6x6": {"device": dev_vox, "host": host_vox, "speedup": dev_vox / host_vox,
                            "note": "device: build + pack + upload of 4096; host: build + pack + upload of 512"},
            "knn_points_500_2000": {"device": dev_knn, "host": host_knn, "speedup": dev_knn / host_knn,
                                    "note": "springs only (point sampling and materials on the host in both)"}}


DEVO_ROBOTS, DEVO_K = 512, 128
SG_CHILDREN, SG_WARMUP_BATCHES, SG_RACE_S = 4096, 13, 4.0
# the surrogate's top 35 % of the new children (plus a 5 % audit) is
# simulated: the best 10 % of all children is then found at a rate of
# 0.93-0.96 (copies of simulated genomes, about a fifth of the children and
# two thirds of the best 10 %, take their known fitness), the best 10 % of
# the new children at 0.77-0.85
SG_SCREEN = 0.35


def surrogate_bench(local_rank, generations: int = 8, plain_generations: int = 3, seed: int = 0):
    """Surrogate-screened evolution (4096 children of 6x6x6 voxel genomes
    per generation; copies of simulated genomes take their known fitness,
    and of the new children the surrogate's top 35% plus a 5% random audit
    are simulated for 1 s on land) against plain evolution (every new child
    simulated), after a warm-up of 13 x 4096 = 53,248 simulated genomes
    (3 random batches, then plain-evolution children).  First a race: both
    methods from the warm-up's pool for the same wall-time budget (best
    fitness against time).  Generations/s from host wall time per generation (children,
    screening, device builds, simulation, online training) over timed
    generations after one untimed warm-up generation per method; the screen's
    quality from every child of the screened generations also simulated,
    outside the timed region."""
    import copy
    from mercury_b200 import evolve
    from mercury_b200.surrogate import Surrogate
    ev = evolve.Evaluator(local_rank)
    sg = Surrogate(local_rank, max_batch=1024, seed=seed)
    scr = evolve.ScreenedEvolution(ev, sg, seed=seed + 1, children=SG_CHILDREN, screen=SG_SCREEN)
    warm = scr.warmup(SG_WARMUP_BATCHES * SG_CHILDREN, batch=SG_CHILDREN)
    plain = evolve.PlainEvolution(ev, seed=seed + 2, children=SG_CHILDREN, pool=copy.deepcopy(scr.pool),
                                  memo=copy.deepcopy(scr.memo))
    # best fitness against wall time, both from the pool the warm-up left,
    # for the same budget (one untimed generation each first: a new batch
    # size plans its packing once)
    rs = evolve.ScreenedEvolution(ev, sg, seed=seed + 3, children=SG_CHILDREN, screen=SG_SCREEN)
    rs.data, rs.pool, rs.mu, rs.sd = scr.data, copy.deepcopy(scr.pool), scr.mu, scr.sd
    rs.memo = copy.deepcopy(scr.memo)
    rp = evolve.PlainEvolution(ev, seed=seed + 4, children=SG_CHILDREN, pool=copy.deepcopy(scr.pool),
                               memo=copy.deepcopy(scr.memo))
    start_best = float(scr.pool.fitness[0])
    curves = evolve.race({"screened": rs, "plain": rp}, SG_RACE_S)
    race = {"budget_s": SG_RACE_S, "start_best": start_best, "curves": curves,
            "best_at_budget": {k: evolve.best_at(v, SG_RACE_S) for k, v in curves.items()},
            "note": "both from the warm-up's elite pool; elapsed = sum of generation wall times"}
    # one untimed generation per method first: a new batch size plans its
    # packing once (warm-up, like the headline's warm-up steps)
    warm_s = scr.generation(truth=True)
    warm_p = plain.generation()
    gens = [scr.generation(truth=True) for _ in range(generations)]
    pgens = [plain.generation() for _ in range(plain_generations)]
    t_s = float(np.mean([g["wall_s"] for g in gens]))
    t_p = float(np.mean([g["wall_s"] for g in pgens]))
    q = {k: float(np.mean([g[k] for g in gens])) for k in ("spearman", "top10_recall", "top10_recall_new",
                                                          "top10_recall_top10", "random_screen_recall",
                                                          "known_share", "known_in_top10")}
    # recall of the screen's top fraction alone (no audit), per fraction
    q["top10_recall_at"] = {fr: float(np.mean([g["top10_recall_at"][fr] for g in gens]))
                            for fr in gens[0]["top10_recall_at"]}

    def rounded(g):
        return {k: ({a: round(b, 4) for a, b in v.items()} if isinstance(v, dict) else round(v, 4))
                for k, v in g.items()}
    return {"metric": "generations/s", "screened": 1.0 / t_s, "plain": 1.0 / t_p, "speedup": t_p / t_s,
            "unit": "generations/s", **q,
            "per_generation": [rounded(g) for g in gens],
            "plain_per_generation": [rounded(g) for g in pgens],
            "best_fitness": {"screened": gens[-1]["best"], "plain": pgens[-1]["best"]},
            "race": race,
            "warmup": warm, "warmup_generation_s": {"screened": warm_s["wall_s"], "plain": warm_p["wall_s"]},
            "simulated_per_generation": {"screened": float(np.mean([g["simulated"] for g in gens])),
                                         "plain": float(np.mean([g["simulated"] for g in pgens]))},
            "workload": f"{SG_CHILDREN} children of 6x6x6 voxel genomes per generation, 1 s on land "
                        f"(dt 1e-4, 10,000 steps); copies of simulated genomes take their known fitness "
                        f"(both methods), screen {round(100 * SG_SCREEN)}% + 5% audit of the new children; warm-up "
                        f"{SG_WARMUP_BATCHES * SG_CHILDREN} simulated genomes (3 random batches, then "
                        f"plain-evolution children)"}


def devo_population():
    """DevoBenchmark's population (optimize/benchmark.cpp:171-217): copies of
    the reference's default VoxelRobot (VoxelRobot::Initialize,
    VoxelRobot.cpp:352-381: 12^3 points, bone inside, air on the upper
    faces; 1,728 masses, 18,788 springs)."""
    import mercury_b200 as mb
    from mercury_b200 import robots
    grid = np.full((12, 12, 12), 22, np.uint8)
    grid[11, :, :] = grid[:, 11, :] = grid[:, :, 11] = 0
    e = robots.lattice_robot(grid, 1.0)
    return mb.pack([e] * DEVO_ROBOTS)


def devo_bench(local_rank, calls=3):
    """Springs replaced per second by Devo() with the reference's default
    replaced_springs_per_element (128, config.h:18) on 512 default robots,
    after 100 stress-tracked steps; wall time of the synchronous call,
    median of 3 calls (the first call on a population also sets up the
    device re-packing).  The robots are too large for one CTA: development
    runs on the device on the streamed layout and on the split layout (the
    default for stepping such robots; their parts are re-derived with the
    partition kept), timed beside it."""
    import mercury_b200 as mb

    def run(cfg, n_calls):
        b = devo_population()
        sim = mb.Simulator(local_rank)
        sim.setTimeStep(1e-4)
        sim.set_launch_config(**cfg)
        sim.set_batch(b)
        sim.run_steps(100, True)
        sim.synchronize()
        walls, phases = [], []
        for i in range(n_calls):
            t0 = time.perf_counter()
            n = sim.devo(DEVO_K, i)
            walls.append(time.perf_counter() - t0)
            phases.append(sim.devo_profile())
        w = float(np.median(walls))
        ph = phases[int(np.argsort(walls)[len(walls) // 2])]
        sim.run_steps(1000, True)  # the rewired population keeps stepping
        return n, w, ph, not sim.robot_flags().any(), sim.launch_config()

    n, w, ph, finite, cfg = run({"cluster": 1}, calls)
    _, ws, phs, fin_s, cfg_s = run({}, calls)
    return {"metric": "springs replaced/s", "value": n / w, "unit": "springs/s", "replaced_per_call": n,
            "ms_per_call": 1e3 * w, "phases": ph, "finite_after": finite and fin_s,
            "workload": f"{DEVO_ROBOTS} default voxel robots (1,728 masses, 18,788 springs), "
                        f"{DEVO_K} springs per robot, after 100 tracked steps",
            "path": "streamed" if cfg["streamed"] else "resident",
            "split_layout": {"ms_per_call": 1e3 * ws, "phases": phs, "cluster": cfg_s["cluster"]}}


def run_reference(args, rank, local_rank, world):
    """Reference arm, rank 0 only.  Nothing of the product is loaded here:
    the population is built by the reference's own VoxelRobot::Build
    (oracle/population.py through oracle/_ref), the material table and the
    timed step are the oracle's."""
    if rank != 0:
        return None
    from oracle import core, population
    pop, duration, dt, track = WORKLOADS[args.workload]
    batch = population.population_batch(pop, seed_base=1000 * {"small": 0, "uneven": 1, "streamed": 4}[pop])
    active = batch.active_springs()
    table = core.material_table()
    threads = os.cpu_count() or 1
    steps_total = core.step_count(duration, dt)
    # bounded sample per bench step: all robots, `sample` steps
    p, v = batch.pos.copy(), batch.vel.copy()
    s = np.zeros(batch.n_springs, np.float32)
    t0 = time.perf_counter()
    core.xpbd_run(batch, p, v, s, table, dt, 0.0, 10, track, threads)
    rate = active * 10 / max(time.perf_counter() - t0, 1e-9)
    sample = int(max(10, min(steps_total, 4.0 * rate / active)))
    for _ in range(args.warmup):
        p, v = batch.pos.copy(), batch.vel.copy()
        core.xpbd_run(batch, p, v, s, table, dt, 0.0, min(sample, 10), track, threads)
    tt = 0.0
    for _ in range(args.steps):
        p, v = batch.pos.copy(), batch.vel.copy()
        s[:] = 0
        t0 = time.perf_counter()
        core.xpbd_run(batch, p, v, s, table, dt, 0.0, sample, track, threads)
        tt += time.perf_counter() - t0
    value = active * sample * args.steps / tt
    ref_cuda = ref_devo = None
    if not args.no_ref_cuda:
        try:
            ref_cuda = reference_cuda(batch, dt, duration, track)
        except Exception as e:  # the reference's GPU path is optional evidence
            ref_cuda = {"unavailable": str(e)[:200]}
        try:
            ref_devo = reference_devo()
        except Exception as e:
            ref_devo = {"unavailable": str(e)[:200]}
    return {
        "impl": "reference",
        "metric": "spring-updates/s",
        "value": value,
        "unit": "spring-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * tt / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.workload}: {batch.n_robots} voxel robots, {active} non-air springs, "
                               f"reference XPBD step, dt={dt}, {duration} s = {steps_total} steps per "
                               f"evaluation; the rate is per spring-update, measured on a bounded sample "
                               f"of {sample} of those steps for all robots per bench step",
                   "parallelism": "CPU, OpenMP over robots",
                   "robots": "built by the reference's VoxelRobot::Build (oracle/_ref)"},
        "cpu_baseline": {"value": value, "unit": "spring-updates/s", "cores": threads, "kind": "port",
                         "sample": f"all {batch.n_robots} robots x {sample} of {steps_total} steps per bench step"},
        "e2e": {"value": value, "unit": "spring-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": ref_cuda,
        "reference_cuda_devo": ref_devo,
    }


def _ref_lib():
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libmercury_ref.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.ref_decode_id.argtypes = [ctypes.c_uint32]
    L.ref_decode_id(1)
    return L


def reference_cuda(batch, dt, duration, track):
    """The reference's own CUDA simulator (oracle/_ref, built from its
    sources) on the same population.  `value` times Simulate(duration) alone
    on the host clock, as optimize/benchmark.cpp:96-99 does (Simulate
    synchronises after every launch); `wall_*` adds SetElements (host
    packing, allocation, H2D) and Collect (D2H)."""
    import ctypes
    L = _ref_lib()
    if L is None:
        return {"unavailable": "oracle/_ref/libmercury_ref.so not built"}
    L.ref_simulate_timed.argtypes = ([ctypes.c_int] + [ctypes.c_void_p] * 8 +
                                     [ctypes.c_float, ctypes.c_float, ctypes.c_int] + [ctypes.c_void_p] * 3)
    L.ref_simulate_timed.restype = ctypes.c_int
    mo = batch.mass_offsets.astype(np.int32)
    so = batch.spring_offsets.astype(np.int32)
    pos3 = np.ascontiguousarray(batch.pos[:, :3])
    vel3 = np.ascontiguousarray(batch.vel[:, :3])
    po, vo = np.zeros_like(pos3), np.zeros_like(vel3)
    secs = np.zeros(2, np.float64)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    args = (batch.n_robots, P(mo), P(pos3), P(vel3), P(batch.mass_material), P(so),
            P(np.ascontiguousarray(batch.pairs)), P(batch.lbar), P(batch.spring_material))
    short = min(duration, 0.01)
    L.ref_simulate_timed(*args, dt, short, int(track), P(po), P(vo), P(secs))  # warm-up
    steps = L.ref_simulate_timed(*args, dt, duration, int(track), P(po), P(vo), P(secs))
    active = batch.active_springs()
    return {"value": active * steps / secs[0], "unit": "spring-updates/s", "steps": steps,
            "simulate_s": float(secs[0]), "value_all_springs": batch.n_springs * steps / secs[0],
            "wall_value": active * steps / secs[1], "wall_s": float(secs[1]),
            "note": "value: Simulate alone (4 launches and 4 syncs per step), host clock, as the reference's "
                    "benchmark times it; wall_value: SetElements + Simulate + Collect; masses padded per "
                    "robot to the largest count"}


def reference_devo(calls=3):
    """The reference's Simulator::Devo (oracle/_ref) on the population of
    devo_bench (copies of the reference's default robot, built by its own
    VoxelRobot::Build), timed per call on the host clock as DevoBenchmark
    does."""
    import ctypes
    from oracle import population
    L = _ref_lib()
    if L is None:
        return {"unavailable": "oracle/_ref/libmercury_ref.so not built"}
    pos, mm, pairs, lbar, sm, _, _ = population.build_cells(np.full((11, 11, 11), population.BONE, np.uint8), 1.0)
    R = DEVO_ROBOTS
    nm, ns = len(pos), len(lbar)
    mo = (np.arange(R + 1) * nm).astype(np.int32)
    so = (np.arange(R + 1) * ns).astype(np.int32)
    pos3 = np.ascontiguousarray(np.tile(pos, (R, 1)))
    vel3 = np.zeros_like(pos3)
    L.ref_devo_time.argtypes = ([ctypes.c_int] + [ctypes.c_void_p] * 8 +
                                [ctypes.c_uint, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_void_p])
    L.ref_devo_time.restype = ctypes.c_int
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    secs = np.zeros(calls, np.float64)
    L.ref_devo_time(R, P(mo), P(pos3), P(vel3), P(np.tile(mm, R)), P(so),
                    P(np.ascontiguousarray(np.tile(pairs, (R, 1)))), P(np.tile(lbar, R)), P(np.tile(sm, R)),
                    DEVO_K, 1e-4, 0.01, calls, P(secs))
    w = float(np.median(secs))
    n = DEVO_ROBOTS * DEVO_K
    return {"metric": "springs replaced/s", "value": n / w, "unit": "springs/s", "ms_per_call": 1e3 * w,
            "calls_ms": [1e3 * x for x in secs],
            "note": "Simulator::Devo after Simulate(0.01 s, track): CUB segmented sort (with its own "
                    "cudaMalloc/cudaFree), cuRAND pairs, replaceSprings; host clock per call"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="uneven", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the force-mode, streamed and devo lines")
    ap.add_argument("--autotune-cache", action="store_true",
                    help="reuse (and store) the autotuner's choice in its cache file instead of re-tuning")
    args = ap.parse_args()

    rank, local_rank, world = (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
                               int(os.environ.get("WORLD_SIZE", 1)))
    if args.impl == "reference":  # loads nothing of the product
        if rank != 0:
            return
        line = run_reference(args, rank, local_rank, world)
        print(json.dumps(line), flush=True)
        return
    from mercury_b200 import dist
    dist.init("nccl" if world > 1 else "gloo")
    try:
        line = run_ours(args, rank, local_rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.finalize()


if __name__ == "__main__":
    main()
