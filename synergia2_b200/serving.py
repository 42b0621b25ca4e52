"""Continuous-batching request loop for tracking jobs.

Jobs (lattice, bunch, grid, turns) arrive over time.  The server admits
queued jobs in arrival order while the device memory they need fits in its
budget and keeps every admitted bunch and its space-charge workspace
resident on the GPU.  Each admitted job runs on its own CUDA stream in
quanta of turns (sized so that jobs of unequal cost per turn hold the GPU
for similar amounts of work; one CUDA graph per turn): the loop launches a
job's next quantum as soon as its previous one has finished, so the work of
all active jobs overlaps on the device, and a finished job is retired and
its memory handed to the next arrival without waiting for the others.  Job
latency is completion time minus arrival time.
"""
import dataclasses
import time
from dataclasses import dataclass, field

import numpy as np

from . import (Batch, Bunch, Four_momentum, Lattice, Lattice_element, Propagator, Reference_particle,
               Space_charge_3d_open_hockney_options, Split_operator_stepper, pconstants, precision_t)


@dataclass
class JobSpec:
    job_id: int
    lattice: list            # element dicts {type, name, double: {...}}
    steps_per_turn: int      # split-operator steps (space-charge kicks) per turn
    n: int                   # macroparticles
    grid: tuple              # (gx, gy, gz)
    turns: int
    sigmas: tuple            # (x, xp, y, yp, cdt, dpop)
    seed: int
    arrival: float = 0.0     # seconds after the stream starts
    kinetic_energy: float = 2.5
    real_num: float = 1e11


@dataclass
class JobResult:
    job_id: int
    arrival: float
    admitted: float
    completed: float
    n: int
    turns: int
    steps: int
    emittance: np.ndarray = field(default=None)
    particles: np.ndarray = field(default=None)

    @property
    def latency(self):
        return self.completed - self.arrival


def footprint_bytes(spec, precision=precision_t.mixed):
    """Device memory of one admitted job: particles (7 FP64 columns, mask,
    discard flag) and their cell-ordered working copy (two more copies and
    two index arrays), and the space-charge workspace."""
    gx, gy, gz = spec.grid
    nx, ny, nz = 2 * gx, 2 * gy, 2 * gz
    G = gx * gy * gz
    nkxp = (nx // 2 + 2) & ~1
    spec_bytes = nz * ny * nkxp * (8 if precision == precision_t.mixed else 16)
    e_bytes = G * (16 if precision == precision_t.mixed else 32)
    phi_bytes = G * (4 if precision == precision_t.mixed else 8)
    rho_bytes = G * (4 if precision == precision_t.mixed else 8)
    ghat = (nx // 2 + 1) * (ny // 2 + 1) * (nz // 2 + 1) * 8
    return spec.n * (3 * 58 + 8) + rho_bytes + spec_bytes + e_bytes + phi_bytes + ghat + (1 << 20)


def make_lattice(elements, kinetic_energy):
    fm = Four_momentum(pconstants.mp)
    fm.set_kinetic_energy(kinetic_energy)
    ref = Reference_particle(1, fm)
    lat = Lattice("job")
    for e in elements:
        le = Lattice_element(e["type"], e["name"])
        for k, v in e.get("double", {}).items():
            le.set_double_attribute(k, v)
        for k, v in e.get("string", {}).items():
            le.set_string_attribute(k, v)
        lat.append(le)
    lat.set_reference_particle(ref)
    return lat, ref


class Server:
    def __init__(self, hbm_budget, max_active=64, precision=precision_t.mixed, graphs=True,
                 quantum_work=2e8, keep_particles=False):
        self.budget = hbm_budget
        self.max_active = max_active
        self.precision = precision
        self.graphs = graphs
        self.quantum_work = quantum_work  # macroparticle-steps per job per iteration (target)
        self.keep_particles = keep_particles
        self.batch = Batch()
        self.active = {}   # slot -> (spec, propagator, bunch, turns_left, admitted)
        self.used = 0
        self.max_inflight = 0  # most jobs with work on the device at once

    def _admit(self, spec, now):
        lat, ref = make_lattice(spec.lattice, spec.kinetic_energy)
        opts = Space_charge_3d_open_hockney_options(*spec.grid)
        opts.precision = self.precision
        prop = Propagator(lat, Split_operator_stepper(opts, spec.steps_per_turn))
        if self.graphs:
            prop.set_graphs(True)
        bunch = Bunch(ref, spec.n, spec.real_num)
        bunch.populate_gaussian(spec.sigmas, spec.seed)
        slot = self.batch.add(prop, bunch)
        self.active[slot] = [spec, prop, bunch, spec.turns, now]
        self.used += footprint_bytes(spec, self.precision)

    def _retire(self, slot, now, results):
        spec, prop, bunch, _, admitted = self.active.pop(slot)
        self.batch.remove(slot)
        emit = bunch.moments()[2]
        parts = bunch.get_particles()[0] if self.keep_particles else None
        results.append(JobResult(spec.job_id, spec.arrival, admitted, now, spec.n, spec.turns,
                                 spec.turns * spec.steps_per_turn, emit, parts))
        self.used -= footprint_bytes(spec, self.precision)
        del prop, bunch

    def run(self, jobs, realtime=True, poll_s=2e-4):
        """Serve `jobs` (JobSpec with arrival offsets in seconds); returns
        (results, wall seconds).  realtime=False ignores the arrival offsets
        (every job is queued at time 0).  The clock is the wall clock from
        the start of the call, so admission (allocation, bunch population)
        is part of every job's latency and of the wall time."""
        if not realtime:
            jobs = [dataclasses.replace(j, arrival=0.0) for j in jobs]
        queue = sorted(jobs, key=lambda j: (j.arrival, j.job_id))
        results = []
        t0 = time.perf_counter()

        def clock():
            return time.perf_counter() - t0

        def arrival(spec):
            return spec.arrival

        inflight = {}  # slot -> turns launched

        def launch_idle():
            # every admitted job that is not running gets its next quantum
            for slot, (spec, _, _, left, _) in self.active.items():
                if slot in inflight or left <= 0:
                    continue
                per_turn = spec.n * spec.steps_per_turn
                q = max(1, min(left, int(self.quantum_work // max(per_turn, 1))))
                self.batch.launch(slot, q)
                inflight[slot] = q
            self.max_inflight = max(self.max_inflight, len(inflight))

        qi = 0
        while qi < len(queue) or self.active:
            now = clock()
            # admission in arrival order while slots and device memory allow;
            # each admitted job starts at once, so its work overlaps the
            # admission of the next
            while qi < len(queue) and arrival(queue[qi]) <= now and len(self.active) < self.max_active:
                need = footprint_bytes(queue[qi], self.precision)
                if self.active and self.used + need > self.budget:
                    break
                self._admit(queue[qi], now)
                qi += 1
                launch_idle()
            launch_idle()
            # collect finished quanta; retire finished jobs at once
            progressed = False
            for slot in list(inflight):
                if self.batch.query(slot):
                    q = inflight.pop(slot)
                    self.active[slot][3] -= q
                    progressed = True
                    if self.active[slot][3] <= 0:
                        self._retire(slot, clock(), results)
            if not progressed:
                if not self.active and qi < len(queue):
                    wait = arrival(queue[qi]) - clock()
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                else:
                    time.sleep(poll_s)
        return results, clock()


def poisson_arrivals(n, rate, seed):
    g = np.random.Generator(np.random.Philox(seed))
    return np.cumsum(g.exponential(1.0 / rate, n))


def summarize(results, wall):
    lat = np.array([r.latency for r in results])
    work = sum(r.n * r.steps for r in results)
    return {"jobs": len(results), "wall_s": wall, "macroparticle_steps": work,
            "throughput": work / wall if wall > 0 else 0.0,
            "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None}
