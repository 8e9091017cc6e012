"""Python mirror of the reference's class Simulator
(common/simulator/Simulator.h:19-149) over the C ABI.

Method names, arguments and defaults follow the reference so that its
callers read the same:

    sim = Simulator()
    sim.Initialize(SimulatorConfig(time_step=1e-3))
    trackers = sim.SetElements(elements)
    sim.Simulate(1.0, trackStresses=False)
    results = sim.Collect(trackers)

Differences, by design: robots may have different mass counts (the
reference requires equal counts, Simulator.cu:231); errors raise
MercuryError instead of exiting the process (Simulator.cu:10-18); Collect
also returns spring stresses (the reference copies them but drops them,
Simulator.cu:540); CentreOfMass() reduces on the device.
"""
from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import _lib
from .element import Batch, Element, pack, unpack
from .materials import material_table

ENVIRONMENT_LAND, ENVIRONMENT_WATER = 0, 1

MODE_REF_XPBD, MODE_FORCE_LAND, MODE_FORCE_WATER = 0, 1, 2

# Environments of the force-based benchmark configurations (land: g, the
# reference's floor stiffness 1e6 (environment.h:15-22), mu_s 1.0, mu_k 0.8;
# water: buoyancy cancels gravity, 0.5 rho Cd A = 0.5 * 1000 * 1 * 1e-4);
# velocity damping 0.999 per step.  No face drag: the benchmark robots carry
# no faces.  WATER_FACES drags on the robots' surface triangles instead of
# per mass, with the density of water.
LAND = dict(g=9.81, floor_stiffness=1.0e6, friction_static=1.0, friction_kinetic=0.8, drag=0.0,
            damping=0.999, face_drag=0.0)
WATER = dict(g=0.0, floor_stiffness=0.0, friction_static=0.0, friction_kinetic=0.0,
             drag=0.5 * 1000.0 * 1.0 * 1e-4, damping=0.999, face_drag=0.0)
WATER_FACES = dict(WATER, drag=0.0, face_drag=1000.0)


def _desc(batch: Batch) -> "_lib.BatchDesc":
    fo, faces = getattr(batch, "face_offsets", None), getattr(batch, "faces", None)
    return _lib.BatchDesc(
        batch.n_robots, _lib.ptr(batch.mass_offsets), _lib.ptr(batch.pos), _lib.ptr(batch.vel),
        _lib.ptr(batch.mass_material), _lib.ptr(batch.spring_offsets), _lib.ptr(batch.pairs),
        _lib.ptr(batch.spring_material), _lib.ptr(batch.lbar),
        _lib.ptr(fo) if faces is not None else None, _lib.ptr(faces) if faces is not None else None)


@dataclass
class SimulatorConfig:
    """Config::Simulator (common/util/config.h:16-21)."""
    visual: bool = False
    replaced_springs_per_element: int = 128
    time_step: float = 0.005
    env_type: int = ENVIRONMENT_WATER


@dataclass
class ElementTracker:
    """Simulator.h:11-17: which masses and springs of the batch are robot ID."""
    ID: int
    mass_begin: int
    mass_end: int
    spring_begin: int
    spring_end: int


class Simulator:
    def __init__(self, device: int = 0):
        ctx = ctypes.c_void_p()
        _lib.check(_lib.LIB.mb_context_create(device, ctypes.byref(ctx)))
        self._ctx = ctx
        self._batch: Batch | None = None
        self._elements: list[Element] = []
        self.config = SimulatorConfig()
        self._table = material_table()
        self._devo_seed = 0
        self._topology_stale = False
        _lib.check(_lib.LIB.mb_set_materials(self._ctx, _lib.ptr(self._table)), self._ctx)
        # the reference's m_deltaT before Initialize (Simulator.h:55)
        self.setTimeStep(0.0001)

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        lib = getattr(_lib, "LIB", None)  # None during interpreter shutdown
        if ctx and lib is not None:
            lib.mb_context_destroy(ctx)
            self._ctx = None

    # -- Simulator.h:27-48 ------------------------------------------------
    def Initialize(self, config: SimulatorConfig | None = None) -> None:
        self.config = config or SimulatorConfig()
        self.setTimeStep(self.config.time_step)
        self.Reset()

    def SetElement(self, element: Element) -> ElementTracker:
        return self.SetElements([element])[0]

    def SetElements(self, elements: list[Element]) -> list[ElementTracker]:
        batch = pack(elements)
        self.set_batch(batch)
        self._elements = list(elements)
        return [ElementTracker(r, int(batch.mass_offsets[r]), int(batch.mass_offsets[r + 1]),
                               int(batch.spring_offsets[r]), int(batch.spring_offsets[r + 1]))
                for r in range(batch.n_robots)]

    def Simulate(self, sim_duration: float, trackStresses: bool = False, trace: bool = False,
                 tracefile: str = "trace.csv") -> int:
        """Runs sim_duration seconds; returns the number of steps taken."""
        if trace:
            raise NotImplementedError("tracing is not supported; Collect between Simulate calls")
        n = ctypes.c_uint32()
        _lib.check(_lib.LIB.mb_simulate(self._ctx, float(sim_duration), int(bool(trackStresses)),
                                        ctypes.byref(n)), self._ctx)
        return n.value

    def Devo(self) -> None:
        """Simulator::Devo (Simulator.cu:640-668): rewires every robot's
        config.replaced_springs_per_element highest-stress springs (see
        devo()).  The seed counts calls on this simulator from 0, as the
        reference's static counter does."""
        self.devo(self.config.replaced_springs_per_element, self._devo_seed)
        self._devo_seed += 1

    def Collect(self, trackers):
        single = isinstance(trackers, ElementTracker)
        trackers = [trackers] if single else list(trackers)
        pos, vel, stress = self.collect_arrays()
        self._refresh_topology()
        full = unpack(self._batch, pos, vel, stress, self._elements)
        out = [full[t.ID] for t in trackers]
        return out[0] if single else out

    def CollectElement(self, tracker: ElementTracker) -> Element:
        return self.Collect(tracker)

    def getDeltaT(self) -> float:
        return float(_lib.LIB.mb_get_time_step(self._ctx))

    def setTimeStep(self, dt: float) -> None:
        _lib.check(_lib.LIB.mb_set_time_step(self._ctx, float(dt)), self._ctx)

    def getTotalTime(self) -> float:
        return float(_lib.LIB.mb_get_total_time(self._ctx))

    def Reset(self) -> None:
        _lib.check(_lib.LIB.mb_set_total_time(self._ctx, 0.0), self._ctx)

    # -- array-level interface ---------------------------------------------
    def set_mode(self, mode: int) -> None:
        """MODE_REF_XPBD (the reference step), MODE_FORCE_LAND or MODE_FORCE_WATER."""
        _lib.check(_lib.LIB.mb_set_mode(self._ctx, int(mode)), self._ctx)

    def set_environment(self, **kw) -> None:
        env = _lib.Environment()
        _lib.check(_lib.LIB.mb_get_environment(self._ctx, ctypes.byref(env)), self._ctx)
        for k, v in kw.items():
            setattr(env, k, float(v))
        _lib.check(_lib.LIB.mb_set_environment(self._ctx, ctypes.byref(env)), self._ctx)

    def environment(self) -> dict:
        env = _lib.Environment()
        _lib.check(_lib.LIB.mb_get_environment(self._ctx, ctypes.byref(env)), self._ctx)
        return {f: getattr(env, f) for f, _ in env._fields_}

    def set_materials(self, table: np.ndarray) -> None:
        self._table = np.ascontiguousarray(table, np.float32)
        _lib.check(_lib.LIB.mb_set_materials(self._ctx, _lib.ptr(self._table)), self._ctx)

    def set_batch(self, batch: Batch) -> None:
        self._batch = batch
        self._vox_batch_n = None
        self._topology_stale = False
        d = _desc(batch)
        _lib.check(_lib.LIB.mb_set_elements(self._ctx, ctypes.byref(d)), self._ctx)

    def devo(self, replaced_per_robot: int, seed: int, reference_ranks: bool = False) -> int:
        """Development (mb_devo): the springs of stress ranks [0, k) of every
        robot (ranks [r k, r k + k) with reference_ranks) get random mass
        pairs, the composite material of the pair and the mean length at the
        current clock.  Updates the batch's topology; returns the number of
        springs replaced."""
        n = ctypes.c_uint32()
        flags = _lib.DEVO_REFERENCE_RANKS if reference_ranks else 0
        _lib.check(_lib.LIB.mb_devo(self._ctx, int(replaced_per_robot), int(seed), flags,
                                    ctypes.byref(n)), self._ctx)
        self._topology_stale = True  # read back on demand (Collect, batch)
        return n.value

    def _refresh_topology(self) -> None:
        if self._topology_stale:
            pairs, mat, lbar = self.collect_springs()
            mm = np.empty(self._batch.n_masses, np.uint8)
            _lib.check(_lib.LIB.mb_collect_mass_materials(self._ctx, _lib.ptr(mm)), self._ctx)
            self._batch = dataclasses.replace(self._batch, pairs=pairs, spring_material=mat, lbar=lbar,
                                              mass_material=mm)
            self._topology_stale = False

    def set_voxel_population(self, cells: np.ndarray, h: float = 0.1, mass: float = 1.0) -> None:
        """Uploads voxel robots built on the device (mb_set_voxel_population)
        from `cells`, an (R, sx, sy, sz) array of base material ids indexed
        [robot, x, y, z]; the same robots as pack([robots.voxel_robot(c, h,
        mass) for c in cells]) followed by set_batch."""
        cells = np.asarray(cells, np.uint8)
        if cells.ndim != 4:
            raise ValueError("cells must be (robots, sx, sy, sz)")
        R, sx, sy, sz = cells.shape
        flat = np.ascontiguousarray(cells.transpose(0, 3, 2, 1))  # x fastest
        _lib.check(_lib.LIB.mb_set_voxel_population(self._ctx, R, sx, sy, sz, _lib.ptr(flat), float(h),
                                                    float(mass)), self._ctx)
        key = (sx, sy, sz, float(h), float(mass))
        if getattr(self, "_vox_tmpl_key", None) != key:
            from .robots import lattice_robot
            self._vox_tmpl = lattice_robot(np.ones((sx + 1, sy + 1, sz + 1), np.uint8), h, mass)
            self._vox_tmpl_key = key
        t = self._vox_tmpl
        if self._batch is None or getattr(self, "_vox_batch_n", None) != (R, key):
            P, S = t.n_masses, t.n_springs
            pos = np.zeros((R * P, 4), np.float32)
            pos[:, :3] = np.tile(t.pos, (R, 1))
            pos[:, 3] = mass
            self._batch = Batch(np.arange(R + 1, dtype=np.int64) * P, pos, np.zeros((R * P, 4), np.float32),
                                np.zeros(R * P, np.uint8), np.arange(R + 1, dtype=np.int64) * S,
                                np.tile(t.pairs, (R, 1)), np.zeros(R * S, np.uint8),
                                np.tile(t.mean_length, R))
            self._vox_batch_n = (R, key)
        self._elements = [t] * R
        self._topology_stale = True

    @property
    def batch(self) -> Batch:
        """The uploaded population, with the topology as development left it."""
        self._refresh_topology()
        return self._batch

    def devo_profile(self) -> dict:
        """Phases of the last devo(): wall ms of the device part and of a
        host re-pack (0 if none), and the number of host re-packs so far."""
        ms = np.zeros(3, np.float64)
        _lib.check(_lib.LIB.mb_devo_profile(self._ctx, _lib.ptr(ms)), self._ctx)
        return {"device_ms": float(ms[0]), "host_repack_ms": float(ms[1]), "host_repacks": int(ms[2])}

    def collect_springs(self):
        """(pairs (S, 2) uint16, material (S,) uint8, mean length (S,) float32)
        of the population on the device (mb_collect_springs)."""
        S = self._batch.n_springs
        pairs = np.empty((S, 2), np.uint16)
        mat = np.empty(S, np.uint8)
        lbar = np.empty(S, np.float32)
        _lib.check(_lib.LIB.mb_collect_springs(self._ctx, _lib.ptr(pairs), _lib.ptr(mat), _lib.ptr(lbar)),
                   self._ctx)
        return pairs, mat, lbar

    def set_state(self, pos: np.ndarray, vel: np.ndarray) -> None:
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        _lib.check(_lib.LIB.mb_set_state(self._ctx, _lib.ptr(pos), _lib.ptr(vel)), self._ctx)

    def run_steps(self, steps: int, track_stresses: bool = False) -> None:
        _lib.check(_lib.LIB.mb_run_steps(self._ctx, int(steps), int(bool(track_stresses))), self._ctx)

    def collect_arrays(self, out=None):
        b = self._batch
        if b is None:
            raise _lib.MercuryError(4, "no population uploaded")
        if out is None:
            pos = np.empty((b.n_masses, 4), np.float32)
            vel = np.empty((b.n_masses, 4), np.float32)
            stress = np.empty(b.n_springs, np.float32)
        else:
            pos, vel, stress = out
        _lib.check(_lib.LIB.mb_collect(self._ctx, _lib.ptr(pos), _lib.ptr(vel), _lib.ptr(stress)),
                   self._ctx)
        return pos, vel, stress

    def CentreOfMass(self) -> np.ndarray:
        """(R, 3) centre of mass of the non-air masses of every robot."""
        com = np.empty((self._batch.n_robots, 3), np.float32)
        _lib.check(_lib.LIB.mb_centre_of_mass(self._ctx, _lib.ptr(com)), self._ctx)
        return com

    def robot_flags(self) -> np.ndarray:
        f = np.empty(self._batch.n_robots, np.uint32)
        _lib.check(_lib.LIB.mb_robot_flags(self._ctx, _lib.ptr(f)), self._ctx)
        return f

    def synchronize(self) -> None:
        _lib.check(_lib.LIB.mb_synchronize(self._ctx), self._ctx)

    @property
    def stream(self) -> int:
        return int(_lib.LIB.mb_get_stream(self._ctx) or 0)

    def device_state(self):
        p, v, s = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(_lib.LIB.mb_device_state(self._ctx, ctypes.byref(p), ctypes.byref(v),
                                            ctypes.byref(s)), self._ctx)
        return p.value, v.value, s.value

    def launch_config(self) -> dict:
        c = _lib.LaunchConfig()
        _lib.check(_lib.LIB.mb_get_launch_config(self._ctx, ctypes.byref(c)), self._ctx)
        return {f: getattr(c, f) for f, _ in c._fields_}

    def step_variant(self) -> dict:
        """The step kernel the next launches use (mb_get_step_variant):
        register_rows (each mass's row held in registers) and the dynamic
        shared memory per CTA."""
        rr, smem = ctypes.c_uint32(), ctypes.c_uint32()
        _lib.check(_lib.LIB.mb_get_step_variant(self._ctx, ctypes.byref(rr), ctypes.byref(smem)), self._ctx)
        return {"register_rows": rr.value, "smem_bytes": smem.value}

    def packed_springs(self) -> np.ndarray:
        """The packed word of every spring slot on the device, in slot order
        (mb_get_packed_springs): a | b << 12 | material slot << 24."""
        n = ctypes.c_uint64()
        _lib.check(_lib.LIB.mb_get_packed_springs(self._ctx, None, 0, ctypes.byref(n)), self._ctx)
        out = np.empty(n.value, np.uint32)
        _lib.check(_lib.LIB.mb_get_packed_springs(self._ctx, _lib.ptr(out), n.value, ctypes.byref(n)),
                   self._ctx)
        return out

    def set_launch_config(self, threads=0, springs_per_thread=0, masses_per_thread=0, bins=0,
                          chunk=0, use_graph=1, streamed=0, cluster=0) -> None:
        c = _lib.LaunchConfig(threads, springs_per_thread, masses_per_thread, bins, chunk, use_graph,
                              streamed, cluster)
        _lib.check(_lib.LIB.mb_set_launch_config(self._ctx, ctypes.byref(c)), self._ctx)


def fitness(com: np.ndarray, base_com: np.ndarray, length: np.ndarray) -> np.ndarray:
    """SoftBody::updateFitness (SoftBody.cpp:124-137): max((x - x0)/length, 0)."""
    return np.maximum((com[:, 0] - base_com[:, 0]) / length, 0.0).astype(np.float32)


def body_length(batch: Batch) -> np.ndarray:
    """SoftBody::updateLength (SoftBody.cpp:98-110): max(|x_max - x_min|, 1)
    over non-air masses, with both extremes starting at 0."""
    out = np.ones(batch.n_robots, np.float32)
    for r in range(batch.n_robots):
        ms, _ = batch.robot_slices(r)
        x = batch.pos[ms, 0][batch.mass_material[ms] != 0]
        lo = min(0.0, float(x.min())) if x.size else 0.0
        hi = max(0.0, float(x.max())) if x.size else 0.0
        out[r] = max(abs(np.float32(hi) - np.float32(lo)), 1.0)
    return out


def plan(batch: Batch, num_sms: int = 148, smem_bytes: int = 0, **cfg) -> dict:
    """Launch plan of a population computed on the host, without a GPU
    (mb_plan_population): shape, bins, path and packed-layout statistics."""
    d = _desc(batch)
    c = _lib.LaunchConfig(cfg.get("threads", 0), cfg.get("springs_per_thread", 0),
                          cfg.get("masses_per_thread", 0), cfg.get("bins", 0), cfg.get("chunk", 0),
                          cfg.get("use_graph", 1), cfg.get("streamed", 0), cfg.get("cluster", 0))
    st = _lib.PlanStats()
    _lib.check(_lib.LIB.mb_plan_population(ctypes.byref(d), ctypes.byref(c), num_sms, smem_bytes,
                                           ctypes.byref(st)))
    return {f: getattr(st, f) for f, _ in st._fields_}
