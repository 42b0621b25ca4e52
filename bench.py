"""Benchmark: macroparticle-steps/s of the split-operator space-charge +
tracking step on the FODO-cell configuration (4,194,304 macroparticles,
64 x 64 x 128 grid, 8 space-charge kicks per 10 m cell, adaptive domain,
linear Green function, FP64).

A step is one split-operator step of the bunch: first-half maps, the 3D open
Hockney kick, second-half maps.  value = macroparticles alive x steps / time
over all ranks (N GPUs run independent bunches: replicas, weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

N_PART = 4194304
GRID = (64, 64, 128)
KICKS_PER_CELL = 8
SIGMAS = [1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4]
REAL_NUM = 1e11
WORKLOAD = ("FODO cell (QF 0.5 m k1=+0.6, D 4.5 m, QD 0.5 m k1=-0.6, D 4.5 m), 8 space-charge kicks per cell, "
            "2.5 GeV protons, 4,194,304 macroparticles, 6D Gaussian, 3D open Hockney 64x64x128 "
            "(doubled 128x128x256), linear Green function, adaptive domain")


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class Clocks:
    """SM clock and clock-event reasons of this process's GPU sampled during
    the timed region: NVML polled every 2 ms from a thread (a timed region of
    20 steps lasts only ~15 ms), the device matched by PCI bus id; falls back
    to nvidia-smi (200 ms samples) when NVML is unavailable.  Read-only
    queries: nothing about the GPU's settings is changed."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, dev):
        self.dev = dev
        self.p = None
        self.thread = None
        self.samples = []
        self.smax = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.dev)
        bus = "%08x:%02x:%02x.0" % (getattr(props, "pci_domain_id", 0), props.pci_bus_id, props.pci_device_id)
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        try:
            import threading
            nv, h = self._nvml_handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()

            def poll():
                while not self.stop_flag.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        pass
                    time.sleep(0.002)
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            time.sleep(0.005)  # the first sample precedes the timed region
            return
        except Exception:
            self.thread = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=1.0)
            if not self.samples:
                return None
            reasons = set()
            for _, r in self.samples:
                for bit, nm in self.REASONS.items():
                    if r & bit:
                        reasons.add(nm)
            return {"sm_mhz": statistics.median(c for c, _ in self.samples), "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(self.samples), "source": "nvml, 2 ms"}
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            return None
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def fp64_roofline(syn, workload, n, light, full):
    """FP64 side of the particle passes: algorithmic FP64 operations per
    launch (the per-macroparticle counts of profiles/fp64_flops_per_particle.json,
    made by running the oracle's particle code on a counting scalar, times the
    macroparticles) over the measured average launch time, against the FP64
    FMA peak of this GPU measured now.  light / full are (total ms, launches)
    of the two kernel variants over the timed region."""
    path = os.path.join(ROOT, "profiles", "fp64_flops_per_particle.json")
    try:
        w = json.load(open(path))["workloads"][workload]
    except (OSError, KeyError, ValueError):
        return None
    pk = ctypes.c_double()
    syn.check(syn.lib().sb2_fp64_peak_probe(ctypes.byref(pk), None))
    out = {"bound": "fp64", "unit": "TFLOP/s", "peak": pk.value,
           "peak_source": "measured in this run: sb2_fp64_peak_probe, independent FP64 FMA chains on every SM "
                          "(an FMA counts 2)",
           "flops_source": "profiles/fp64_flops_per_particle.json (python oracle/count_flops.py)"}
    for name, (ms, cnt), key in (("full_variant", full, "full_pass_flops_mean"),
                                 ("light_variant", light, "light_pass_flops_mean")):
        if cnt:
            fl = w[key] * n
            ach = fl / (ms / cnt * 1e-3) / 1e12
            out[name] = {"flops_per_particle": w[key], "algorithmic_flops_per_launch": fl,
                         "avg_launch_ms": ms / cnt, "achieved": ach, "frac": ach / pk.value}
    return out


def cpu_baseline_c3(steps=2):
    """The oracle on all host cores for a bounded sample of the ring
    workload: the same 2^24-macroparticle bunch and 128^2 x 256 grid, the
    first `steps` split-operator steps of the turn; one turn (384 steps) and
    100 turns are extrapolated from the per-step time."""
    from helpers import MP, gaussian_bunch, oracle_lattice, ring_cell
    from oracle import oracle as O
    threads = O.set_threads(os.cpu_count() or 1)
    spec = []
    for c in range(24):
        for e in ring_cell(radius=0.05):
            e = dict(e)
            e["name"] = "%s_%d" % (e["name"], c)
            spec.append(e)
    n = 1 << 24
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 3)
    sim = O.Sim(oracle_lattice(spec), n, REAL_NUM, stepper=O.STEPPER_SPLIT, num=16 * 24,
                sc=O.SCOptions.make(128, 128, 256), value=2.5 + MP)
    sim.set_particles(p)
    del p
    t0 = time.perf_counter()
    sim.propagate_steps(0, steps)
    dt = time.perf_counter() - t0
    nv, _, _ = sim.counts()
    return {"value": nv * steps / dt, "unit": "macroparticle-steps/s", "cores": threads, "kind": "port",
            "sample": "%d macroparticles x %d steps (the first of the turn) of the same workload, %.1f s" % (n, steps, dt),
            "one_turn_s_extrapolated": dt / steps * 384, "hundred_turns_h_extrapolated": dt / steps * 38400 / 3600}


def ring_c3(syn, torch, turns=1, warmup_steps=16):
    """Config 3: the 24-cell ring (QF 0.5, SF thin, D 0.75, B 2.0, D 0.75,
    QD 0.5, SD thin, D 0.75, B 2.0, D 0.75 per cell; circular aperture 5 cm on
    every element), 2^24 macroparticles, 128x128x256 grid, 16 kicks per cell
    (384 steps per turn), FP64 and mixed precision, each propagator
    autotuned first; device time with CUDA events per turn."""
    from helpers import product_lattice, ring_cell
    spec = []
    for c in range(24):
        for e in ring_cell(radius=0.05):
            e = dict(e)
            e["name"] = "%s_%d" % (e["name"], c)
            spec.append(e)
    lat, ref = product_lattice(spec)
    n = 1 << 24
    out = {"macroparticles": n, "grid": [128, 128, 256], "steps_per_turn": 384, "turns": turns}
    for prec in ("fp64", "mixed"):
        opts = syn.Space_charge_3d_open_hockney_options(128, 128, 256)
        opts.precision = getattr(syn.precision_t, prec)
        prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 16 * 24))
        bunch = syn.Bunch(ref, n, REAL_NUM)
        bunch.populate_gaussian([2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 3)
        prop.propagate_steps(bunch, 0, warmup_steps)
        best, trials = prop.autotune(bunch, steps=16)
        # graphs per turn segment, captured ahead (untimed)
        prop.set_graphs(True)
        prop.prepare_steps(bunch, warmup_steps, 384 * turns)
        torch.cuda.synchronize()
        L = syn.lib()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        prop.propagate_steps(bunch, warmup_steps, 384 * turns)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        graph_stats = prop.graph_stats()
        prop.set_graphs(False)  # the breakdown launches directly
        alive = bunch.get_total_num()
        emit = [float(x) for x in bunch.moments()[2]]
        # breakdown: the first 96 steps of the next turn with CUDA events
        # around every launch (outside the timed turn)
        nprof = 96
        L.sb2_profile_enable(1)
        for c in range(8):
            L.sb2_profile_read(c, None, None, None, 1)
        prop.propagate_steps(bunch, warmup_steps + 384 * turns, nprof)
        torch.cuda.synchronize()
        L.sb2_profile_enable(0)
        brk, raw = {}, {}
        for c in range(8):
            nm, tot, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_int64()
            syn.check(L.sb2_profile_read(c, ctypes.byref(nm), ctypes.byref(tot), ctypes.byref(cnt), 1))
            brk[nm.value.decode()] = round(tot.value / nprof, 4)
            raw[nm.value.decode()] = (tot.value, cnt.value)
        out[prec] = {"value": alive * 384 * turns / (ms * 1e-3), "ms_per_step": ms / (384 * turns), "alive": alive,
                     "step_breakdown_ms": brk, "emittance": emit,
                     "roofline_fp64": fp64_roofline(syn, "ring_c3", alive, raw.get("track", (0.0, 0)),
                                                    raw.get("track_full", (0.0, 0))),
                     "autotune": {"best": best, "trials": len(trials), "default_ms": round(trials[0]["ms"], 3),
                                  "best_ms": round(min(r["ms"] for r in trials), 3)},
                     "graphs": {"captured_ahead": graph_stats[0], "replayed": graph_stats[1]}}
        del prop, bunch
        torch.cuda.empty_cache()
    out["value"] = out["mixed"]["value"]
    # rms emittances of the two precisions after the same turns from one seed
    out["emittance_rel_diff_xyz"] = [abs(a / b - 1.0) for a, b in zip(out["mixed"]["emittance"],
                                                                     out["fp64"]["emittance"])]
    return out


def fodo_lattice(syn):
    from helpers import MP, fodo_cell, product_lattice
    return product_lattice(fodo_cell())


def c1_propagator(syn, precision, graphs=False):
    lat, ref = fodo_lattice(syn)
    opts = syn.Space_charge_3d_open_hockney_options(*GRID)
    opts.precision = precision
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, KICKS_PER_CELL))
    if graphs:
        prop.set_graphs(True)
    return prop, ref


def _emittances(bunch):
    return [float(e) for e in bunch.moments()[2]]


def mixed_vs_fp64(syn, torch, steps, warmup, passes, seed=1):
    """The FODO workload in mixed precision (FP64 particles and maps, FP32
    spectrum / potential / field): throughput over `steps` steps with CUDA
    events; the field error of one solve of each precision on the same
    particles (the FP64 run's state after `passes` passes); the relative
    rms-emittance difference per plane after `passes` passes from one
    seed."""
    fp64, mixed = syn.precision_t.fp64, syn.precision_t.mixed
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    prop, ref = c1_propagator(syn, mixed)
    b = syn.Bunch(ref, N_PART, REAL_NUM)
    b.populate_gaussian(SIGMAS, seed=seed)
    prop.propagate_steps(b, 0, warmup, stream=sp)
    prop.set_graphs(True)  # as the FP64 headline: graphs per turn segment, captured ahead
    prop.prepare_steps(b, warmup, steps, stream=sp)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    prop.propagate_steps(b, warmup, steps, stream=sp)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    rate = b.get_total_num() * steps / (ms * 1e-3)
    del prop, b

    ends, emits = [], []
    for prec in (fp64, mixed):
        prop, ref = c1_propagator(syn, prec)
        b = syn.Bunch(ref, N_PART, REAL_NUM)
        b.populate_gaussian(SIGMAS, seed=seed)
        prop.propagate(b, passes)
        emits.append(_emittances(b))
        ends.append(b)
        del prop
    e64, e32 = emits
    demit = [abs(a / c - 1.0) for a, c in zip(e32, e64)]

    # field error: both precisions solve on the FP64 run's final particles
    parts, masks, _ = ends[0].get_particles()
    fields = []
    for prec in (fp64, mixed):
        opts = syn.Space_charge_3d_open_hockney_options(*GRID)
        opts.precision = prec
        bb = syn.Bunch(ends[0].reference_particle, N_PART, REAL_NUM)
        bb.set_particles(parts, masks)
        sc = syn.Space_charge_3d_open_hockney(opts)
        sc.apply(bb, 1.25 / (ends[0].reference_particle.get_beta() * 299792458.0))
        fields.append(sc.last())
        del sc, bb
    num = sum(float(((fields[1][c] - fields[0][c]) ** 2).sum()) for c in ("ex", "ey", "ez"))
    den = sum(float((fields[0][c] ** 2).sum()) for c in ("ex", "ey", "ez"))
    return {"value": rate, "unit": "macroparticle-steps/s", "ms_per_step": ms / steps,
            "precision": "mixed (FP64 particles, maps and Green function; FP32 charge grid from exact fixed-point tile sums; FP32 spectrum, potential, field; FP64 butterflies)",
            "field_rel_l2": math.sqrt(num / den), "field_tol": 1e-5,
            "emittance_rel_diff_xyz": demit, "emittance_tol": 1e-4, "passes": passes}


def stream_jobs(syn, njobs, seed, ring_fraction, nmax, turns_max, grids, rate):
    """Seeded tracking jobs drawn as the served-stream workload: lattice the
    FODO cell (8 kicks per turn) or the 24-cell ring (16 kicks per cell,
    384 per turn) with probability `ring_fraction`; macroparticles
    log-uniform in [5e4, nmax]; grid uniform over `grids`; turns uniform in
    [1, turns_max]; Gaussian bunch with sigma_x,y uniform in [0.5, 3] mm;
    Poisson arrivals at `rate` jobs/s."""
    import numpy as np
    from helpers import fodo_cell, ring_cell
    from synergia2_b200.serving import JobSpec, poisson_arrivals
    g = np.random.Generator(np.random.Philox(seed))
    arrivals = poisson_arrivals(njobs, rate, seed + 1)
    jobs = []
    for i in range(njobs):
        ring = g.uniform() < ring_fraction
        n = int(math.exp(g.uniform(math.log(5e4), math.log(nmax))))
        grid = grids[int(g.integers(len(grids)))]
        turns = int(g.integers(1, turns_max + 1))
        sx, sy = g.uniform(0.5e-3, 3e-3, 2)
        sig = (float(sx), 1e-4, float(sy), 1e-4, 0.3, 1e-4)
        lattice = ring_cell() * 24 if ring else fodo_cell()
        jobs.append(JobSpec(job_id=i, lattice=lattice, steps_per_turn=384 if ring else 8, n=n, grid=tuple(grid),
                            turns=turns, sigmas=sig, seed=1000 + i, arrival=float(arrivals[i])))
    return jobs


def served_stream(syn, njobs, seed, ring_fraction=0.0, nmax=2e6, turns_max=10,
                  grids=((32, 32, 64), (64, 64, 128)), rate=1e9):
    """The same seeded job stream (same arrival times) served twice: by the
    continuous-batching server (mixed precision, CUDA-graph turns, up to 64
    jobs resident and overlapping, admission by device-memory footprint) and
    by the plain FP64 path one job at a time in arrival order.  Throughput =
    macroparticle-steps of all jobs / wall time from the first arrival to
    the last completion, admission and bunch population included."""
    from synergia2_b200.serving import Server, summarize
    out = {"jobs": njobs, "ring_fraction": ring_fraction, "n_range": [5e4, nmax], "turns_max": turns_max,
           "grids": [list(g) for g in grids], "arrival_rate_per_s": rate, "unit": "macroparticle-steps/s"}
    jobs = stream_jobs(syn, njobs, seed, ring_fraction, nmax, turns_max, grids, rate)
    srv = Server(hbm_budget=100 << 30, max_active=64)
    res, wall = srv.run(jobs, realtime=True)
    served = summarize(res, wall)
    jobs = stream_jobs(syn, njobs, seed, ring_fraction, nmax, turns_max, grids, rate)
    seq = Server(hbm_budget=1 << 40, max_active=1, precision=syn.precision_t.fp64, graphs=False)
    res, wall = seq.run(jobs, realtime=True)
    plain = summarize(res, wall)
    out.update({"served_throughput": served["throughput"], "latency_p50_s": served["latency_p50_s"],
                "latency_p99_s": served["latency_p99_s"], "wall_s": served["wall_s"],
                "macroparticle_steps": served["macroparticle_steps"],
                "plain_fp64_throughput": plain["throughput"], "plain_fp64_latency_p50_s": plain["latency_p50_s"],
                "plain_fp64_latency_p99_s": plain["latency_p99_s"], "plain_fp64_wall_s": plain["wall_s"],
                "speedup_vs_plain_fp64": served["throughput"] / plain["throughput"]})
    return out


def batched_scan(syn, torch, nbunches, passes, seed, lockstep=True):
    """Quad-strength scan: `nbunches` independent bunches (k1 uniform in
    [0.4, 0.8], macroparticles log-uniform in [1e5, 4e6], grid drawn from
    32^2x64, 64^2x128, 64^2x256), mixed precision, all advanced together by
    one Batch: in lockstep (one work-list launch per kernel kind and grid
    shape per step for all bunches) or with a stream and CUDA-graph turns
    per bunch; throughput over `passes` passes after one warm-up pass."""
    import numpy as np
    from helpers import fodo_cell, product_lattice
    g = np.random.Generator(np.random.Philox(seed))
    grids = [(32, 32, 64), (64, 64, 128), (64, 64, 256)]
    batch = syn.Batch()
    keep = []
    for i in range(nbunches):
        k1 = float(g.uniform(0.4, 0.8))
        n = int(math.exp(g.uniform(math.log(1e5), math.log(4e6))))
        grid = grids[int(g.integers(3))]
        lat, ref = product_lattice(fodo_cell(k1))
        opts = syn.Space_charge_3d_open_hockney_options(*grid)
        opts.precision = syn.precision_t.mixed
        prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, KICKS_PER_CELL))
        prop.set_graphs(not lockstep)
        b = syn.Bunch(ref, n, REAL_NUM)
        b.populate_gaussian(SIGMAS, seed=10 + i)
        keep.append((prop, b, batch.add(prop, b)))
    slots = [s for _, _, s in keep]

    def advance(turns):
        if lockstep:
            batch.run_lockstep(slots, turns)
        else:
            batch.run({s: turns for s in slots})
    advance(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    advance(passes)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    alive = sum(b.get_total_num() for _, b, _ in keep)
    total = sum(b.size() for _, b, _ in keep)
    return {"bunches": nbunches, "macroparticles": total, "passes": passes, "precision": "mixed",
            "mode": "lockstep work lists" if lockstep else "stream and CUDA-graph turns per bunch",
            "value": alive * passes * KICKS_PER_CELL / dt, "unit": "macroparticle-steps/s", "wall_s": dt}


def algorithmic_bytes_per_step(n, grid, w=8):
    """Per step: one fused particle pass (6 FP64 columns in and out, mask +
    discards) and one deposit pass (x, y, cdt), plus each grid array moved
    once: 3G + 8S words (rho, rho-hat, G-hat refresh, phi; E formed in the
    kick)."""
    gx, gy, gz = grid
    G = gx * gy * gz
    S = (gx + 1) * (2 * gy) * (2 * gz)
    return n * (96 + 24 + 3) + w * (3 * G + 8 * S), n * (96 + 2)


def cpu_baseline(steps=KICKS_PER_CELL):
    """The oracle (CPU FP64 restatement of the reference) on all host cores:
    the same bunch size and grid, one FODO cell (8 steps)."""
    from helpers import MP, fodo_cell, gaussian_bunch, oracle_lattice
    from oracle import oracle as O
    threads = O.set_threads(os.cpu_count() or 1)
    p = gaussian_bunch(N_PART, SIGMAS, 1)
    sim = O.Sim(oracle_lattice(fodo_cell()), N_PART, REAL_NUM, stepper=O.STEPPER_SPLIT, num=KICKS_PER_CELL,
                sc=O.SCOptions.make(*GRID), value=2.5 + MP)
    sim.set_particles(p)
    t0 = time.perf_counter()
    sim.propagate_steps(0, steps)
    dt = time.perf_counter() - t0
    nv, _, _ = sim.counts()
    return {"value": nv * steps / dt, "unit": "macroparticle-steps/s", "cores": threads, "kind": "port",
            "sample": "%d macroparticles x %d steps (one FODO cell) of the same workload, %.1f s" %
                      (N_PART, steps, dt)}


def run_reference(args, rank):
    """Reference arm: the oracle port of the reference's CPU path (the
    reference itself cannot be built here: Kokkos/MPI/FFTW absent) on all
    host cores, the same 4,194,304-macroparticle bunch and grid, one
    split-operator step per timed step."""
    if rank != 0:
        return
    from helpers import MP, fodo_cell, gaussian_bunch, oracle_lattice
    from oracle import oracle as O
    threads = O.set_threads(os.cpu_count() or 1)
    n = N_PART
    p = gaussian_bunch(n, SIGMAS, 1)
    sim = O.Sim(oracle_lattice(fodo_cell()), n, REAL_NUM, stepper=O.STEPPER_SPLIT, num=KICKS_PER_CELL,
                sc=O.SCOptions.make(*GRID), value=2.5 + MP)
    sim.set_particles(p)
    sim.propagate_steps(0, args.warmup)
    t0 = time.perf_counter()
    sim.propagate_steps(args.warmup, args.steps)
    dt = time.perf_counter() - t0
    nv, _, _ = sim.counts()
    v = nv * args.steps / dt
    sample = "%d macroparticles per step, 64x64x128 grid, %d steps, %.1f s" % (n, args.steps, dt)
    print(json.dumps({"impl": "reference", "metric": "macroparticle-steps/s", "value": v,
                      "unit": "macroparticle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": WORKLOAD, "sample": sample},
                      "cpu_baseline": {"value": v, "unit": "macroparticle-steps/s", "cores": threads,
                                       "kind": "port", "sample": sample},
                      "e2e": {"value": v, "unit": "macroparticle-steps/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}))


def over_ranks(dist, torch, seconds, work, device):
    """Whole-job timing over replicas: the slowest rank's time and the sum
    of all ranks' work (macroparticle-steps)."""
    if dist is None:
        return seconds, work
    t = torch.tensor([float(seconds)], device=device, dtype=torch.float64)
    w = torch.tensor([float(work)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return t.item(), w.item()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=80)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="time the default launch shapes")
    ap.add_argument("--no-graphs", action="store_true", help="time direct launches instead of CUDA-graph turns")
    ap.add_argument("--particles", type=int, default=N_PART, help="bunch size (profiling cases only)")
    ap.add_argument("--config", default="c1", choices=["c1", "c2", "c3", "c4"],
                    help="c1: FODO 4M FP64 + mixed (default); c2: 64-bunch quad scan; c3: 24-cell ring, 2^24 "
                         "macroparticles, 128^2x256; c4: served job stream")
    ap.add_argument("--extras", type=int, default=1, help="0: skip the mixed-precision and served legs of c1")
    ap.add_argument("--jobs", type=int, default=48, help="c4: jobs in the served stream")
    ap.add_argument("--turns", type=int, default=1, help="c3: turns of the ring per precision")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    if args.config in ("c2", "c3", "c4"):
        # single-GPU workloads: rank 0 alone runs them
        import synergia2_b200 as syn
        if rank == 0:
            if args.config == "c3":
                r = ring_c3(syn, torch, turns=args.turns)
                if not args.no_cpu_baseline:
                    r["cpu_baseline"] = cpu_baseline_c3()
                wl = ("24-cell ring (QF, SF thin, B 2 m, QD, SD thin; circular aperture 5 cm), 2^24 macroparticles, "
                      "128^2x256 grid, 16 kicks per cell, one turn (384 steps) in FP64 and in mixed precision")
            elif args.config == "c2":
                r = batched_scan(syn, torch, 64, 50, seed=7, lockstep=True)
                r["streams_and_graphs"] = batched_scan(syn, torch, 64, 50, seed=7, lockstep=False)
                wl = ("quad-strength scan: 64 FODO bunches, k1 U[0.4,0.8], macroparticles log-uniform [1e5,4e6], "
                      "grids {32^2x64, 64^2x128, 64^2x256}, 50 passes, mixed precision, advanced in lockstep "
                      "(one work-list launch per kernel kind and grid shape per step)")
            else:
                r = served_stream(syn, args.jobs, seed=11, ring_fraction=0.5, nmax=8e6, turns_max=50,
                                  grids=((32, 32, 64), (64, 64, 128), (128, 128, 256)), rate=4.0)
                wl = ("served stream: %d jobs (Poisson arrivals 4/s), FODO cell or 24-cell ring (p=0.5), "
                      "macroparticles log-uniform [5e4,8e6], grids {32^2x64, 64^2x128, 128^2x256}, turns U[1,50]"
                      % args.jobs)
            v = r.get("value", r.get("served_throughput"))
            print(json.dumps({"metric": "macroparticle-steps/s", "value": v, "unit": "macroparticle-steps/s",
                              "n_gpus": 1, "higher_is_better": True, "dtype": "f64 particles / f32 grid",
                              "data": "synthetic", "config": {"workload": wl}, "result": r}))
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import synergia2_b200 as syn
    from helpers import MP
    L = syn.lib()
    syn.check(L.sb2_set_device(local))  # the library's own (static) CUDA runtime
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    lat, ref = fodo_lattice(syn)
    opts = syn.Space_charge_3d_open_hockney_options(*GRID)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, KICKS_PER_CELL))
    npart = args.particles
    bunch = syn.Bunch(ref, npart, REAL_NUM)
    bunch.populate_gaussian(SIGMAS, seed=1 + rank)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    prop.propagate_steps(bunch, 0, args.warmup, stream=sp)
    barrier()

    # the project's autotuner picks the particle-pass launch shapes and the
    # re-sort interval on a scratch copy of the bunch (untimed)
    # (48 steps, six FODO cells, per trial: with shorter trials run-to-run
    # noise of about 1% picks the candidate)
    tuned = None
    if not args.no_autotune:
        best, trials = prop.autotune(bunch, steps=48)
        tuned = {"best": best, "trials": len(trials), "steps_per_trial": 48,
                 "default_ms": round(trials[0]["ms"], 3), "best_ms": round(min(r["ms"] for r in trials), 3)}
    barrier()

    # CUDA-graph turns: the steps of the K that fall in one turn are one
    # graph launch; the graphs are captured ahead, untimed, without running
    # anything
    if not args.no_graphs:
        prop.set_graphs(True)
        prop.prepare_steps(bunch, args.warmup, args.steps, stream=sp)
    barrier()

    # timed region: device time with CUDA events on the launching stream
    # (the library's per-category profiler is off: its event pairs around
    # every launch would be timed too)
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    prop.propagate_steps(bunch, args.warmup, args.steps, stream=sp)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    n_alive = bunch.get_total_num()
    graph_stats = prop.graph_stats()
    prop.set_graphs(False)  # the breakdown and the e2e leg launch directly

    # the same K steps once more with the per-category profiler (CUDA events
    # around every launch on the launching stream): the step breakdown and
    # the kernels' launch times of the rooflines
    L.sb2_profile_enable(1)
    for c in range(8):
        L.sb2_profile_read(c, None, None, None, 1)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    p0.record(stream)
    prop.propagate_steps(bunch, args.warmup + args.steps, args.steps, stream=sp)
    p1.record(stream)
    barrier()
    L.sb2_profile_enable(0)
    prof_ms = p0.elapsed_time(p1)
    prof = {}
    for c in range(8):
        nm, tot, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_int64()
        syn.check(L.sb2_profile_read(c, ctypes.byref(nm), ctypes.byref(tot), ctypes.byref(cnt), 1))
        prof[nm.value.decode()] = (tot.value, cnt.value)

    t_max, total_steps = over_ranks(dist, torch, ms, n_alive * args.steps, "cuda")
    value = total_steps / (t_max * 1e-3)

    # end to end through the public API with host buffers: checkin from pinned
    # host memory, K steps in one propagate call with every step's bunch
    # counts copied to pinned host memory as the step completes
    # (sb2_propagator_set_step_counts), checkout to pinned host memory.
    host = torch.empty((7, npart), dtype=torch.float64, pin_memory=True)
    hmask = torch.empty(npart, dtype=torch.uint8, pin_memory=True)
    pd = ctypes.cast(host.data_ptr(), ctypes.POINTER(ctypes.c_double))
    pm = ctypes.cast(hmask.data_ptr(), ctypes.POINTER(ctypes.c_uint8))
    syn.check(L.sb2_bunch_get_particles(bunch.h, pd, pm, None))
    e2e_steps = 0 if args.no_e2e else args.steps
    prop.set_step_counts(max(e2e_steps, 1))  # pinned: written by the device at a device-side cursor
    if e2e_steps and not args.no_graphs:
        # graph turns here too: the timed call starts with a check-in of these
        # host arrays; the same check-in, untimed, lets prepare_steps derive
        # and capture that call's graphs (nothing runs on the GPU)
        prop.set_graphs(True)
        syn.check(L.sb2_bunch_set_particles(bunch.h, pd, pm))
        prop.prepare_steps(bunch, args.warmup + 2 * args.steps, e2e_steps, stream=sp)
    e2e_g0 = prop.graph_stats()
    barrier()
    t0 = time.perf_counter()
    syn.check(L.sb2_bunch_set_particles(bunch.h, pd, pm))
    if e2e_steps:
        syn.check(L.sb2_propagator_propagate_steps(prop.h, bunch.h, args.warmup + 2 * args.steps, e2e_steps, sp))
    syn.check(L.sb2_bunch_get_particles(bunch.h, pd, pm, None))
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    step_counts = prop.step_counts()
    e2e_graphs = tuple(a - b for a, b in zip(prop.graph_stats(), e2e_g0))
    prop.set_graphs(False)
    prop.set_step_counts(0)
    if len(step_counts) != e2e_steps:
        raise RuntimeError("per-step counts: %d records for %d steps" % (len(step_counts), e2e_steps))
    e2e_total = sum(c[1] for c in step_counts) if e2e_steps else bunch.get_total_num()
    e2e_s, e2e_total = over_ranks(dist, torch, e2e_s, e2e_total, "cuda")
    bunch_bytes = npart * (7 * 8 + 1)

    if rank == 0:
        pk, src = peaks()
        # dominant HBM-bound kernel: the light particle pass (drifts, thin
        # kicks, apertures, the space-charge kick); the full pass (Yoshida
        # quadrupole slices) is bound by the FP64 pipe and reported beside it
        tr_ms, tr_n = prof.get("track", (0.0, 0))
        tf_ms, tf_n = prof.get("track_full", (0.0, 0))
        alg_step, alg_track = algorithmic_bytes_per_step(n_alive, GRID)
        achieved = alg_track / ((tr_ms / max(tr_n, 1)) * 1e-3) / 1e9 if tr_n else 0.0
        traffic = None
        tf = os.path.join(ROOT, "profiles", "track_traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get("light_bytes_per_launch")
            except Exception:
                traffic = None
        gpu_launches = int(tr_n + tf_n + prof.get("domain", (0, 0))[1] + prof.get("deposit", (0, 0))[1] +
                           4 * prof.get("green", (0, 0))[1] + 5 * prof.get("solve", (0, 0))[1] +
                           prof.get("efield", (0, 0))[1] + 5 * prof.get("sort", (0, 0))[1])
        out = {
            "metric": "macroparticle-steps/s", "value": value, "unit": "macroparticle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if npart == N_PART else WORKLOAD.replace("4,194,304", str(npart)),
                       "global_batch": npart * world, "grid": list(GRID),
                       "precision": "fp64 (drop-in)", "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (bunch 235 MB per GPU)",
                       "launch": ("CUDA graphs, one per turn or part of a turn inside the K steps (%d captured "
                                  "ahead, untimed; %d replayed)" % graph_stats)
                       if not args.no_graphs else "direct launches",
                       "step_breakdown_ms": {k: round(v[0] / args.steps, 4) for k, v in prof.items()},
                       "step_breakdown_how": "a second run of the same K steps, direct launches with CUDA events "
                                             "around every launch (%.4f ms/step with those events)"
                                             % (prof_ms / args.steps)},
            "roofline": {"kernel": "track_kernel light variant (fused particle pass)", "bound": "hbm",
                         "achieved": achieved, "peak": pk["hbm_gbs"], "peak_source": src, "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg_track,
                         "launches": tr_n, "avg_launch_ms": tr_ms / max(tr_n, 1),
                         "full_variant": {"bound": "fp64 pipe", "launches": tf_n,
                                          "avg_launch_ms": tf_ms / max(tf_n, 1)},
                         "fp64": fp64_roofline(syn, "fodo_c1", n_alive, (tr_ms, tr_n), (tf_ms, tf_n))},
            "e2e": {"value": e2e_total / e2e_s, "unit": "macroparticle-steps/s",
                    "h2d_bytes_per_step": bunch_bytes / args.steps,
                    "d2h_bytes_per_step": bunch_bytes / args.steps + 16,
                    "how": "checkin from pinned host, K steps in one C-ABI propagate call with each step's bunch "
                           "counts written to pinned host by the device as the step completes, checkout to pinned "
                           "host" + ("; CUDA graphs per turn segment captured ahead (untimed), %d captured and %d replayed in "
                                     "the call" % e2e_graphs if not args.no_graphs and args.steps and not args.no_e2e else "")},
            "gpu_launches": gpu_launches,
            "autotune": tuned,
            "clocks": clk,
        }
        if args.extras and world == 1 and npart == N_PART:
            out["mixed"] = mixed_vs_fp64(syn, torch, args.steps, args.warmup, passes=100)
            # a sample of the served-stream configuration: its job mix, sizes,
            # grids and turns, Poisson arrivals
            out["served"] = served_stream(syn, 16, seed=11, ring_fraction=0.5, nmax=8e6, turns_max=50,
                                          grids=((32, 32, 64), (64, 64, 128), (128, 128, 256)), rate=4.0)
        if not args.no_cpu_baseline and world == 1 and npart == N_PART:
            out["cpu_baseline"] = cpu_baseline()
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
