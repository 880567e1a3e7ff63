"""The 32^3 dam break against its golden record (`golden/c1_dam_break_32k.json`,
made by `golden/make_c1_golden.py` from the oracle).

The record holds the FNV-1a hash over (x, v) of every particle, in original
order, after 1, 10, 100 and 1000 steps. The CPU test checks that the oracle
still reproduces the early records; the GPU test checks that the product's
step reproduces all of them, i.e. stays bit-identical to the oracle for 1000
steps (tolerance: exact bits).
"""
import json
import os

import pytest

import oracle as O
import physics_engine_rs as pe
from helpers import dam_break_params_pe, product_dam_break

HERE = os.path.dirname(os.path.abspath(__file__))
DT = 1e-4


def _golden():
    with open(os.path.join(HERE, "golden", "c1_dam_break_32k.json")) as f:
        return json.load(f)


def test_oracle_reproduces_golden_early_steps():
    g = _golden()
    w = O.World(O.dam_break_scene(32), O.dam_break_params(materialize=False))
    done = 0
    for s in (1, 10):
        w.run(DT, s - done)
        done = s
        rec = g["records"][str(s)]
        assert f"{w.hash64():016x}" == rec["hash64"], s
        x = w.x()
        assert [float(c).hex() for c in x[0]] == rec["x_first"]


@pytest.mark.gpu
def test_product_reproduces_golden_1000_steps():
    g = _golden()
    p = product_dam_break(32, 32, 32)
    assert len(p) == g["particles"]
    w = pe.WcsphWorld(p, dam_break_params_pe(), pe.WcsphConfig(use_graph=True))
    done = 0
    for s in sorted(int(k) for k in g["records"]):
        w.run(DT, s - done)
        done = s
        rec = g["records"][str(s)]
        got = w.diagnostics()["hash64"]
        assert f"{got:016x}" == rec["hash64"], f"step {s}"
        assert w.t == rec["t"]
    w.close()
