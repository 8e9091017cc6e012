"""One launch of the step kernel on a named population, for profilers.

    python -m mercury_b200.profile_case [--population uneven] [--steps 1000]
        [--track] [--threads T --spt S --mpt M] [--bins B] [--water-faces]

--water-faces: the water mode with the face drag on robots carrying their
surface triangles (0.1 kg masses), instead of the reference step.

Uploads the population, runs one warm-up launch of `steps` steps, then the
launch to profile (ncu: -k regex:step_kernel -s 1 -c 1), and prints the
device time of the second launch.
"""
from __future__ import annotations

import argparse
import time

import mercury_b200 as mb
from mercury_b200 import robots


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--population", default="uneven")
    ap.add_argument("--robots", type=int, default=None)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--dt", type=float, default=1e-4)
    ap.add_argument("--track", action="store_true")
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--spt", type=int, default=0)
    ap.add_argument("--mpt", type=int, default=0)
    ap.add_argument("--bins", type=int, default=0)
    ap.add_argument("--water-faces", action="store_true")
    args = ap.parse_args()
    faces = args.water_faces
    batch = robots.population_batch(args.population, args.robots, mass=0.1 if faces else 1.0, faces=faces)
    sim = mb.Simulator(0)
    if faces:
        from mercury_b200 import simulator as S
        sim.set_materials(mb.materials.force_table())
        sim.set_mode(S.MODE_FORCE_WATER)
        sim.set_environment(**S.WATER_FACES)
    sim.setTimeStep(args.dt)
    sim.set_launch_config(args.threads, args.spt, args.mpt, args.bins, chunk=args.steps, use_graph=0)
    sim.set_batch(batch)
    sim.run_steps(args.steps, args.track)
    sim.synchronize()
    t0 = time.perf_counter()
    sim.run_steps(args.steps, args.track)
    sim.synchronize()
    el = time.perf_counter() - t0
    act = batch.active_springs()
    print(f"{args.population}: {batch.n_robots} robots, {act} active springs, config {sim.launch_config()}, "
          f"{args.steps} steps in {el * 1e3:.2f} ms wall -> {act * args.steps / el:.3e} spring-updates/s")


if __name__ == "__main__":
    main()
