"""Extract golden tracking vectors from the synergia2 reference's own libFF tests.

Run once with SYNERGIA_REF set to the root of a synergia2 checkout (read
only); writes tests/golden/madx_tracks.json, which the tests read on any
machine:

    SYNERGIA_REF=<synergia2 checkout> python tests/golden/make_golden.py

Sources (paths inside the synergia2 project):
  src/synergia/libFF/tests/test_madx_elements.cc:10-16,100-230   fixture,
      16-particle initial state, de_to_dp, tolerances (1e-10; quad_long 1e-8;
      cdt 100x looser)
  src/synergia/libFF/tests/test_madx_multipoles.cc:86-212        multipole
      fixture (positions only), tolerance 1e-15 (combined-function
      sbends 1e-7)
  src/synergia/libFF/tests/lattices/l_*.seq, mpole_*.seq,
      cfsbend_*.seq                                                 element
      definitions
  src/synergia/libFF/tests/lattices/madx_*.out                     MAD-X
      TRACKONE output; rows >= 26 hold the final coordinates, columns 2..7
      are X PX Y PY T PT (read_madx_output in both test files)
  lattice/madx_reader.cc:81,165-178                                 a final
      drift is appended only when sequence length - position > 1e-6
"""
import json
import math
import os
import re
import sys

REF = os.environ.get("SYNERGIA_REF")
if not REF and __name__ == "__main__":
    sys.exit("set SYNERGIA_REF to the root of a synergia2 checkout")
LAT = os.path.join(REF or "", "src/synergia/libFF/tests/lattices")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "madx_tracks.json")

P0 = 1.5
MP = 0.938272046  # physical_constants.h PDG 2012


def de_to_dp(de):
    return math.sqrt(1 + de * de + 2 * de * math.sqrt(P0 * P0 + MP * MP) / P0) - 1.0


def parse_value(txt, env):
    txt = txt.strip()
    if txt.startswith("{"):
        return [parse_value(t, env) for t in txt.strip("{}").split(",")]
    return float(eval(txt, {"__builtins__": {}}, dict(env, pi=math.pi)))


def split_top(s):
    """Split on commas that are not inside braces."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    out.append(cur)
    return out


def parse_seq(path):
    env, elements, seq_len = {}, {}, None
    text = open(path).read()
    for stmt in [s.strip() for s in text.split(";") if s.strip()]:
        m = re.match(r"^(\w+)\s*=\s*(.+)$", stmt)
        if m and ":" not in stmt:
            env[m.group(1)] = parse_value(m.group(2), env)
            continue
        m = re.match(r"^(\w+)\s*:\s*(\w+)\s*(,.*)?$", stmt, re.S)
        if m:
            label, etype, rest = m.group(1), m.group(2), m.group(3) or ""
            attrs = {}
            for part in split_top(rest)[1:]:
                k, v = part.split("=", 1)
                attrs[k.strip()] = v.strip()
            if etype == "sequence":
                seq_len = parse_value(attrs["l"], env)
                continue
            d = {"type": etype, "name": label, "double": {}, "vector": {}}
            for k, v in attrs.items():
                val = parse_value(v, env)
                if isinstance(val, list):
                    d["vector"][k] = val
                else:
                    d["double"][k] = val
            elements[label] = d
    assert len(elements) == 1, path
    el = list(elements.values())[0]
    lattice = [el]
    if seq_len is None:  # "machine: line=(...)": no sequence length, no tail drift
        return lattice
    tail = seq_len - el["double"].get("l", 0.0)
    if tail > 1.0e-6:
        lattice.append({"type": "drift", "name": "auto_drift", "double": {"l": tail}, "vector": {}})
    return lattice


def read_madx_output(name):
    rows = []
    with open(os.path.join(LAT, "madx_" + name + ".out")) as f:
        for r, line in enumerate(f):
            if r >= 26:
                vals = [float(v) for v in line.split()]
                rows.append(vals[2:8])
    assert len(rows) == 16, name
    return rows


def ring_positions(offset=1.0e-3):
    s2o2 = math.sqrt(2.0) / 2.0
    s3o2 = math.sqrt(3.0) / 2.0
    xy = [(offset, 0.0), (offset * s3o2, offset * 0.5), (offset * s2o2, offset * s2o2),
          (offset * 0.5, offset * s3o2), (0.0, offset), (-offset * 0.5, offset * s3o2),
          (-offset * s2o2, offset * s2o2), (-offset * s3o2, offset * 0.5), (-offset, 0.0),
          (-offset * s3o2, -offset * 0.5), (-offset * s2o2, -offset * s2o2),
          (-offset * 0.5, -offset * s3o2), (0.0, -offset), (offset * 0.5, -offset * s3o2),
          (offset * s2o2, -offset * s2o2), (offset * s3o2, -offset * 0.5)]
    return [[x, 0.0, y, 0.0, 0.0, 0.0] for x, y in xy]


def nllens_golden():
    """src/synergia/libFF/tests/lattices/track_nllensone.npy and
    nllens_channel.seq (README.nllens.txt): 32 particles -- the 16-point ring
    of radius 1 mm around the axis and the same ring around (0.5, -0.25) mm,
    zero angles -- after the thin nonlinear lens (knll 5.479576037e-6, cnll
    8.105461952e-3) between two 0.5 um drifts.  No reference test reads this
    file; its angles are the analytic Danilov-Nagaitsev kick (principal
    square root, asin(z)/(1 - z^2)^(3/2)), which the reference's
    nllens_unit does not compute (tests/test_nllens.py)."""
    import numpy as np
    a = np.load(os.path.join(LAT, "track_nllensone.npy"))
    init = ring_positions() + [[0.5e-3 + r[0], 0.0, -0.25e-3 + r[2], 0.0, 0.0, 0.0] for r in ring_positions()]
    out = os.path.join(os.path.dirname(OUT), "nllens_track.json")
    json.dump({"generated_by": "tests/golden/make_golden.py",
               "source": "src/synergia/libFF/tests/lattices/track_nllensone.npy, nllens_channel.seq",
               "knll": 5.479576037e-06, "cnll": 0.008105461952, "drift": 0.5e-6,
               "initial": init, "final": a.tolist()}, open(out, "w"), indent=0)
    print("wrote", out)


def main():
    cases = []
    # test_madx_elements.cc: drift, quad, sext, quad_long (1e-8), sext_long,
    # octupole, kickers, rf cavity, solenoid (:248-320)
    for name, tol in [("drift", 1e-10), ("quad", 1e-10), ("sext", 1e-10), ("quad_long", 1e-8),
                      ("sext_long", 1e-10), ("oct", 1e-10), ("oct_long", 1e-10), ("kicker", 1e-10),
                      ("hkicker", 1e-10), ("vkicker", 1e-10), ("kicker_long", 1e-10), ("hkicker_long", 1e-10),
                      ("vkicker_long", 1e-10), ("solenoid", 1e-10), ("rfc", 1e-10)]:
        lattice = parse_seq(os.path.join(LAT, "l_" + name + ".seq"))
        for el in lattice:  # the fixture sets cdt_use_drift on every element (:32-33)
            el["double"]["cdt_use_drift"] = 1.0
        init = ring_positions()
        dp = de_to_dp(0.05)
        for p in range(4):
            init[p][1], init[p][3], init[p][4], init[p][5] = 0.01, 0.015, -0.01, dp
        madx = read_madx_output(name)
        expect = [[r[0], r[1], r[2], r[3], -r[4], de_to_dp(r[5])] for r in madx]
        cases.append({"name": name, "lattice": lattice, "p0": P0, "initial": init,
                      "expected": expect, "tol": [tol, tol, tol, tol, tol * 100, tol],
                      "source": "src/synergia/libFF/tests/test_madx_elements.cc"})
    # test_madx_multipoles.cc: mpole_k1..k6 (+ _tilt, s), tolerance 1e-15
    for k in range(1, 7):
        for suf in ("", "_tilt", "s"):
            name = "mpole_k%d%s" % (k, suf)
            lattice = parse_seq(os.path.join(LAT, name + ".seq"))
            madx = read_madx_output(name)
            expect = [[r[0], r[1], r[2], r[3], -r[4], r[5]] for r in madx]
            cases.append({"name": name, "lattice": lattice, "p0": P0, "initial": ring_positions(),
                          "expected": expect, "tol": [1e-15] * 6,
                          "source": "src/synergia/libFF/tests/test_madx_multipoles.cc"})
    # test_madx_multipoles.cc:194-212: combined-function sector bends,
    # tolerance 1e-7
    for name in ("cfsbend_dipole", "cfsbend_dipole_skew", "cfsbend_sext", "cfsbend_sext_skew"):
        lattice = parse_seq(os.path.join(LAT, name + ".seq"))
        madx = read_madx_output(name)
        expect = [[r[0], r[1], r[2], r[3], -r[4], r[5]] for r in madx]
        cases.append({"name": name, "lattice": lattice, "p0": P0, "initial": ring_positions(),
                      "expected": expect, "tol": [1e-7] * 6,
                      "source": "src/synergia/libFF/tests/test_madx_multipoles.cc"})
    nllens_golden()
    json.dump({"generated_by": "tests/golden/make_golden.py", "cases": cases}, open(OUT, "w"), indent=0)
    print("wrote", OUT, len(cases), "cases")


if __name__ == "__main__":
    sys.exit(main())
