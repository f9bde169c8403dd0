"""Extract the golden vectors the tests pin against from the reference tree.

Reads (never copies wholesale) the vendored benchmark tables of the reference
and writes the few numbers the tests use into tests/golden/*.json:

* love_M3L70V01.json: elastic and fluid loading Love numbers h, l, k of the
  M3-L70-V01 earth, degrees 1..64, from data/benchmarks/love_M3-L70-V01/
  mod_M3-L70-V01 (normal-mode table; parsed as tests/test_benchmark_love.f90
  read_ref does: 5 model lines, then per degree a header `n nmodes k h l`,
  nmodes mode lines, and the fluid line `n nmodes k h l`).
* disc_spada2011.json: vertical displacement u and geoid n of the Spada-2011
  disc load at colatitude 0 and on the 0..20 deg profile, at t = 0, 1, 2, 5,
  10 kyr (data/benchmarks/disc_spada2011/{u,n}_disc.txt, 201 rows x 6 times).

* rotation_spada2011.json: Spada-2011 Test 3/2 polar motion |m| [deg] of the
  cap and disc Heaviside loads, Chandler wobble excluded (the quasi-static
  column a time-domain solver targets, TABOO "Gs" values), at t = 0, 1, 2, 5,
  10, 20 kyr, and the published rigid (2,1) geometrical factors G, from
  data/benchmarks/rotation_spada2011/polar_motion_test3-2.txt (rows
  `load cw t m_Vb m_Gs ...`, G in the header comment).

* martinec2018.npz: the Martinec et al. (2018) benchmark profiles of
  data/benchmarks/sle_martinec2018/ as float32 (the tables are float32
  output): A_fig10 (case A cap loading, all 721 rows: colatitude, uplift,
  horizontal, geoid) and {C2,D3,E2,F1}_fig{10..13} (the sea-level cases, every
  second row of the 7 columns: profile coordinate, u, th- and ph-horizontal,
  potential increment -N g, sea surface, sea level).

Run where the reference tree is available, passing its root:
    python tests/golden/make_golden.py <path to the reference tree>
"""
import json
import os
import sys

import numpy as np


def love(ref):
    fn = os.path.join(ref, "data/benchmarks/love_M3-L70-V01/mod_M3-L70-V01")
    lines = open(fn).read().split("\n")[5:]
    out = {"elastic": {}, "fluid": {}}
    i = 0
    while i < len(lines):
        t = lines[i].split()
        if len(t) < 5:
            break
        n, nm = int(t[0]), int(t[1])
        k, h, l = map(float, t[2:5])
        if n <= 64:
            out["elastic"][n] = {"h": h, "l": l, "k": k}
        t = lines[i + 1 + nm].split()
        k, h, l = map(float, t[2:5])
        if n <= 64:
            out["fluid"][n] = {"h": h, "l": l, "k": k}
        i += nm + 2
    return out


def disc(ref):
    d = os.path.join(ref, "data/benchmarks/disc_spada2011")
    u = np.loadtxt(os.path.join(d, "u_disc.txt"))
    n = np.loadtxt(os.path.join(d, "n_disc.txt"))
    return {"theta_deg": [0.1 * i for i in range(201)], "times_kyr": [0, 1, 2, 5, 10, 100],
            "u": u[:, :5].tolist(), "n": n[:, :1].tolist()}


def rotation(ref):
    import re

    fn = os.path.join(ref, "data/benchmarks/rotation_spada2011/polar_motion_test3-2.txt")
    out = {"t_kyr": [], "m_deg": {"cap": [], "disc": []}, "G": {}}
    for line in open(fn):
        if line.startswith("#"):
            g = re.match(r"#\s+(cap|disc)\s*:\s*-\(([0-9.e+-]+)\s*\+\s*i\s*([0-9.e+-]+)\)", line)
            if g:
                out["G"][g.group(1)] = [-float(g.group(2)), -float(g.group(3))]
            continue
        t = line.split()
        if len(t) >= 5 and t[0] in ("cap", "disc") and t[1] == "excl":
            out["m_deg"][t[0]].append(float(t[4]))
            if t[0] == "cap":
                out["t_kyr"].append(float(t[2]))
    return out


def martinec(ref):
    import glob

    d = os.path.join(ref, "data/benchmarks/sle_martinec2018")
    out = {"A_fig10": np.loadtxt(os.path.join(d, "A_fig10_SBK.dat")).astype(np.float32)}
    for fn in sorted(glob.glob(os.path.join(d, "*_fig1?_SBK.dat"))):
        key = os.path.basename(fn)[: -len("_SBK.dat")]
        if key != "A_fig10":
            out[key] = np.loadtxt(fn)[::2].astype(np.float32)
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: make_golden.py <path to the reference tree>")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    json.dump(love(ref), open(os.path.join(here, "love_M3L70V01.json"), "w"), indent=1)
    json.dump(disc(ref), open(os.path.join(here, "disc_spada2011.json"), "w"))
    json.dump(rotation(ref), open(os.path.join(here, "rotation_spada2011.json"), "w"), indent=1)
    np.savez_compressed(os.path.join(here, "martinec2018.npz"), **martinec(ref))
    print("wrote golden fixtures to", here)
