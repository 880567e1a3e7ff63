"""Generate the 32^3 dam-break golden record from the CPU oracle.

Runs the oracle's order-exact restatement of `WcsphWorld::step`
(wcsph.rs:326-347) on the 32x32x32 dam break (1.0 x 0.4 x 0.6 m tank, dx 0.01,
seeded jitter 1e-4, fixed c0 = 20 m/s, dt 1e-4) and writes, at the listed
steps, the FNV-1a hash over (x, v) of every particle in original order plus a
few f64 reductions, to `c1_dam_break_32k.json` beside this script.

The full 1000-step run takes about half an hour on one CPU core:

    python tests/golden/make_c1_golden.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

import oracle as O  # noqa: E402

STEPS = (1, 10, 100, 1000)
DT = 1e-4


def record(w, nf, mass):
    x, v, rho = w.x(), w.v(), w.rho()
    return {
        "hash64": f"{w.hash64():016x}",
        "t": float(w.t),
        "fluid_com": [float(c) for c in x[:nf].mean(axis=0)],
        "fluid_ke": float(0.5 * mass * (v[:nf] ** 2).sum()),
        "rho_min": float(rho[:nf].min()),
        "rho_max": float(rho[:nf].max()),
        # a few raw values as exact hex floats, to localise a mismatch
        "x_first": [float(c).hex() for c in x[0]],
        "v_first": [float(c).hex() for c in v[0]],
        "x_last_fluid": [float(c).hex() for c in x[nf - 1]],
    }


def main():
    O.build()
    scene = O.dam_break_scene(32)
    nf = 32 ** 3
    mass = O.mass_from_spacing(1000.0, 0.01, 3)
    w = O.World(scene, O.dam_break_params(materialize=False))
    out = {
        "scene": "dam break 32x32x32 fluid on dx 0.01 from (dx,dx,dx), jitter 1e-4 seed 0x5EED5EED, "
                 "1-layer Akinci shell of the 1.0 x 0.4 x 0.6 m tank, h = 2 dx, water() with c0 = 20 "
                 "fixed, g = (0, 0, -9.81), dt = 1e-4",
        "fluid": nf,
        "particles": len(scene),
        "records": {},
    }
    done = 0
    t0 = time.time()
    for s in STEPS:
        w.run(DT, s - done)
        done = s
        out["records"][str(s)] = record(w, nf, mass)
        print(f"step {s}: {out['records'][str(s)]['hash64']} ({time.time() - t0:.0f} s)", flush=True)
        with open(os.path.join(HERE, "c1_dam_break_32k.json"), "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
