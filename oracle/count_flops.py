"""ORACLE — test infrastructure only.

Counts the algorithmic FP64 work per macroparticle of the benchmark
workloads by running the oracle with its counting scalar (orc_flops_*: every
add or subtract, multiply, divide, square root and elementary function of
the reference's per-particle arithmetic, as the oracle restates it), and
writes the table the benchmark's FP64 roofline reads:

    python oracle/count_flops.py        # -> profiles/fp64_flops_per_particle.json

A particle pass of the product runs, between two space-charge solves, the
kick of step k, the second-half maps and apertures of step k, the first-half
maps and apertures of step k+1 and the spatial moments for the domain of
the next solve.  The table gives the flops of each such pass of one lattice
cell, per macroparticle, and which kernel variant runs it: "full" when the
pass holds a Yoshida-integrated element or a sector bend, "light" otherwise.
The deposit is its own kernel and is listed apart.  Counts do not depend on
the grid size, so the space-charge operator is counted on a small grid.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this folder is first on the path and would shadow the package
sys.path[:] = [q for q in sys.path if os.path.abspath(q or ".") != HERE]
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from helpers import MP, fodo_cell, gaussian_bunch, oracle_lattice, ring_cell  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "profiles", "fp64_flops_per_particle.json")
HEAVY = ("quadrupole", "sbend", "thick_other")  # categories the full kernel variant integrates

WORKLOADS = {
    "fodo_c1": dict(lattice="FODO cell (QF 0.5 m, D 4.5 m, QD 0.5 m, D 4.5 m)", cell=fodo_cell,
                    kicks=8, sigmas=[1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4]),
    "ring_c3": dict(lattice="24-cell ring cell (QF, SF thin, D, B 2 m, D, QD, SD thin, D, B 2 m, D = 8 m)",
                    cell=ring_cell, kicks=16, sigmas=[2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4]),
}


def _total(cats):
    return sum(sum(ops.values()) for ops in cats.values())


def _add(a, b):
    return {c: {o: a[c][o] + b[c][o] for o in O.FLOP_OPS} for c in O.FLOP_CATEGORIES}


def _only(cats, names):
    z = {o: 0 for o in O.FLOP_OPS}
    return {c: (cats[c] if c in names else dict(z)) for c in O.FLOP_CATEGORIES}


def count_workload(spec, n=4096, seed=1):
    """Per-step operator records of one cell (two cells are run and the
    second is kept, so the pass that wraps around the cell is complete)."""
    p = gaussian_bunch(n, spec["sigmas"], seed)
    sim = O.Sim(oracle_lattice(spec["cell"]()), n, 1e11, stepper=O.STEPPER_SPLIT, num=spec["kicks"],
                sc=O.SCOptions.make(32, 32, 64), value=2.5 + MP)
    sim.set_particles(p)
    s = np.array(spec["sigmas"])
    r2 = ((p[:, :6] / s) ** 2)[:, [0, 2, 4]].sum(axis=1)
    index = int(np.argmin(r2))  # the particle nearest the bunch centre: inside the grid, never lost
    k = spec["kicks"]
    recs = sim.count_flops(index, 0, 2 * k)
    steps = []
    for st in range(k, 2 * k):
        ops = [(kind, cats) for (s_, kind, cats) in recs if s_ == st]
        assert [o[0] for o in ops] == ["I", "C", "I"], ops
        steps.append({"I1": ops[0][1], "C": ops[1][1], "I2": ops[2][1]})
    return index, steps


def passes_of(steps):
    """The particle passes of one cell: kick_k + I2_k + I1_(k+1) + domain_(k+1)."""
    k = len(steps)
    out = []
    for i in range(k):
        a, b = steps[i], steps[(i + 1) % k]
        cats = _add(_add(_only(a["C"], ("sc_kick",)), a["I2"]), _add(b["I1"], _only(b["C"], ("sc_domain",))))
        heavy = any(sum(cats[c].values()) for c in HEAVY)
        out.append({"after_kick_of_step": i, "variant": "full" if heavy else "light",
                    "flops": _total(cats),
                    "by_category": {c: sum(v.values()) for c, v in cats.items() if sum(v.values())},
                    "by_operation": {o: sum(cats[c][o] for c in O.FLOP_CATEGORIES) for o in O.FLOP_OPS}})
    return out


def main():
    table = {
        "what": "algorithmic FP64 operations per macroparticle of each particle pass of one lattice cell, "
                "counted by running the oracle's particle code on a counting scalar",
        "command": "python oracle/count_flops.py",
        "convention": "add/subtract, multiply, divide, square root and elementary function (asin, sin, cos, "
                      "log, exp) count 1 each; sign changes, comparisons, floor and fabs count 0",
        "workloads": {},
    }
    for name, spec in WORKLOADS.items():
        index, steps = count_workload(spec)
        ps = passes_of(steps)
        light = [p["flops"] for p in ps if p["variant"] == "light"]
        full = [p["flops"] for p in ps if p["variant"] == "full"]
        dep = sum(steps[0]["C"]["sc_deposit"].values())
        table["workloads"][name] = {
            "lattice": spec["lattice"], "kicks_per_cell": spec["kicks"], "counted_particle": index,
            "passes": ps,
            "light_passes": len(light), "full_passes": len(full),
            "light_pass_flops_mean": float(np.mean(light)) if light else 0.0,
            "full_pass_flops_mean": float(np.mean(full)) if full else 0.0,
            "deposit_flops": dep,
            "per_step_flops": (sum(light) + sum(full) + dep * len(ps)) / len(ps),
        }
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as f:
        json.dump(table, f, indent=1)
        f.write("\n")
    for name, w in table["workloads"].items():
        print(name, "light %d x %.0f, full %d x %.0f, deposit %d flops/particle" %
              (w["light_passes"], w["light_pass_flops_mean"], w["full_passes"], w["full_pass_flops_mean"],
               w["deposit_flops"]))


if __name__ == "__main__":
    main()
