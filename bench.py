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
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
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
                "samples": len(sm)}


def fodo_lattice(syn):
    from helpers import MP, fodo_cell, product_lattice
    return product_lattice(fodo_cell())


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
    reference itself cannot be built here: Kokkos/MPI/FFTW absent)."""
    if rank != 0:
        return
    from helpers import MP, fodo_cell, gaussian_bunch, oracle_lattice
    from oracle import oracle as O
    threads = O.set_threads(os.cpu_count() or 1)
    n = N_PART // 8  # bounded per-step sample: 524,288 macroparticles
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
    sample = "%d macroparticles (1/8 of the bunch) per step, 64x64x128 grid, %d steps, %.1f s" % (n, args.steps, dt)
    print(json.dumps({"impl": "reference", "metric": "macroparticle-steps/s", "value": v,
                      "unit": "macroparticle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": WORKLOAD, "sample": sample},
                      "cpu_baseline": {"value": v, "unit": "macroparticle-steps/s", "cores": threads,
                                       "kind": "port", "sample": sample},
                      "e2e": {"value": v, "unit": "macroparticle-steps/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=80)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--particles", type=int, default=N_PART, help="bunch size (profiling cases only)")
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
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import synergia2_b200 as syn
    from helpers import MP
    L = syn.lib()
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

    # timed region: device time with CUDA events on the launching stream
    clocks = Clocks(local)
    L.sb2_profile_enable(1)
    for c in range(7):
        L.sb2_profile_read(c, None, None, None, 1)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    prop.propagate_steps(bunch, args.warmup, args.steps, stream=sp)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    L.sb2_profile_enable(0)
    ms = e0.elapsed_time(e1)
    prof = {}
    for c in range(7):
        nm, tot, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_int64()
        syn.check(L.sb2_profile_read(c, ctypes.byref(nm), ctypes.byref(tot), ctypes.byref(cnt), 1))
        prof[nm.value.decode()] = (tot.value, cnt.value)
    n_alive = bunch.get_total_num()

    t_max = ms
    total_steps = n_alive * args.steps
    if dist is not None:
        t = torch.tensor([ms, float(total_steps)], device="cuda", dtype=torch.float64)
        tm = t.clone()
        dist.all_reduce(tm[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(tm[1:], op=dist.ReduceOp.SUM)
        t_max, total_steps = tm[0].item(), tm[1].item()
    value = total_steps / (t_max * 1e-3)

    # end to end through the public API with host buffers: checkin from pinned
    # host memory, K steps (each returning the bunch counts to the host),
    # checkout to pinned host memory.
    host = torch.empty((7, npart), dtype=torch.float64, pin_memory=True)
    hmask = torch.empty(npart, dtype=torch.uint8, pin_memory=True)
    pd = ctypes.cast(host.data_ptr(), ctypes.POINTER(ctypes.c_double))
    pm = ctypes.cast(hmask.data_ptr(), ctypes.POINTER(ctypes.c_uint8))
    syn.check(L.sb2_bunch_get_particles(bunch.h, pd, pm, None))
    barrier()
    e2e_steps = 0 if args.no_e2e else args.steps
    t0 = time.perf_counter()
    syn.check(L.sb2_bunch_set_particles(bunch.h, pd, pm))
    for k in range(e2e_steps):
        syn.check(L.sb2_propagator_propagate_steps(prop.h, bunch.h, args.warmup + k, 1, sp))
    syn.check(L.sb2_bunch_get_particles(bunch.h, pd, pm, None))
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_total = bunch.get_total_num() * max(e2e_steps, 1)
    if dist is not None:
        t = torch.tensor([e2e_s, float(e2e_total)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        e2e_s, e2e_total = t[0].item(), t[1].item()
    bunch_bytes = npart * (7 * 8 + 1)

    if rank == 0:
        pk, src = peaks()
        # dominant kernel: the fused particle pass
        tr_ms, tr_n = prof.get("track", (0.0, 0))
        alg_step, alg_track = algorithmic_bytes_per_step(n_alive, GRID)
        launches_per_step = max(tr_n / args.steps, 1e-9)
        track_bytes_per_launch = alg_track / launches_per_step
        achieved = track_bytes_per_launch / ((tr_ms / max(tr_n, 1)) * 1e-3) / 1e9 if tr_n else 0.0
        traffic = None
        tf = os.path.join(ROOT, "profiles", "track_traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get("bytes_per_launch_c1")
            except Exception:
                traffic = None
        gpu_launches = int(prof.get("track", (0, 0))[1] + prof.get("domain", (0, 0))[1] +
                           prof.get("deposit", (0, 0))[1] + 4 * prof.get("green", (0, 0))[1] +
                           5 * prof.get("solve", (0, 0))[1] + prof.get("efield", (0, 0))[1] +
                           5 * prof.get("sort", (0, 0))[1])
        out = {
            "metric": "macroparticle-steps/s", "value": value, "unit": "macroparticle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if npart == N_PART else WORKLOAD.replace("4,194,304", str(npart)),
                       "global_batch": npart * world, "grid": list(GRID),
                       "precision": "fp64 (drop-in)", "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (bunch 235 MB per GPU)",
                       "step_breakdown_ms": {k: round(v[0] / args.steps, 4) for k, v in prof.items()}},
            "roofline": {"kernel": "track (fused particle pass)", "bound": "hbm", "achieved": achieved,
                         "peak": pk["hbm_gbs"], "peak_source": src, "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                         "algorithmic_bytes_per_launch": track_bytes_per_launch},
            "e2e": {"value": e2e_total / e2e_s, "unit": "macroparticle-steps/s",
                    "h2d_bytes_per_step": bunch_bytes / args.steps,
                    "d2h_bytes_per_step": bunch_bytes / args.steps + 16,
                    "how": "checkin from pinned host, K steps via the C ABI (bunch counts read back each step), "
                           "checkout to pinned host"},
            "gpu_launches": gpu_launches,
            "clocks": clk,
        }
        if not args.no_cpu_baseline and world == 1 and npart == N_PART:
            out["cpu_baseline"] = cpu_baseline()
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
