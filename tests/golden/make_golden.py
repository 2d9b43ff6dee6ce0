"""Generate tests/golden/cavity4_perturbed.npz and conduction4_perturbed.npz
from the oracle.

The reference ships no golden vectors (no test suite) and cannot be built in
this environment, so the fixture records the oracle's FP64 restatement on a
small seeded case: a 4^3 lid-driven cavity with interior nodes perturbed by
+-20% of the spacing (numpy PCG64 seed 12345) and a seeded Gaussian initial
velocity. It stores the geometry, the graph, both assembled systems of the
first outer iteration, and the fields after five SIMPLE iterations. The
conduction fixture is a 4^3 x 6 tet4 block (interior nodes perturbed by +-20%,
lognormal conductivity sigma 1 projected to nodes, U[0,1] source, T = 0 / 1 on
x = 0 / 1): graph, dual volumes, exposed-face areas, the assembled system at a
seeded random temperature, and the temperature after three steps. Run:

    python -m tests.golden.make_golden
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "cavity4_perturbed.npz")
OUT_COND = os.path.join(HERE, "conduction4_perturbed.npz")


def generate(po):
    from openaccel_b200 import meshgen

    m = meshgen.cavity(4, perturb=0.2, seed=12345)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=12345)
    c = po.FlowCase(m, po.default_settings(mom_rtol=1e-13, pc_rtol=1e-13), U0=U0)
    c.initialize()
    out = {}
    rp, cols = c.graph()
    out["row_ptr"], out["cols"] = rp, cols
    out["vol"] = c.field("vol").copy()
    out["faceArea"] = c.field("faceArea").copy()
    out["A_mom"], out["b_mom"] = c.assemble_momentum()
    out["du"] = c.field("du").copy()
    out["A_pc"], out["b_pc"] = c.assemble_pcorr()
    for _ in range(5):
        c.simple_iteration()
    for k in ["U", "p", "mDot", "gradP", "gradU"]:
        out[k + "_it5"] = c.field(k).copy()
    return out


def generate_conduction(po):
    from openaccel_b200 import meshgen

    m, gamma, src, _ = meshgen.conduction(4, sigma=1.0, seed=4242, perturb=0.2)
    c = po.DiffCase(m, gamma, src, po.default_diff_settings(rtol=1e-14, maxit=5000))
    out = {}
    rp, cols = c.graph()
    out["row_ptr"], out["cols"] = rp, cols
    out["vol"] = c.field("vol").copy()
    out["faceArea"] = c.field("faceArea").copy()
    rng = np.random.Generator(np.random.PCG64(99))
    phi0 = rng.uniform(0.0, 1.0, m.nn)
    out["phi0"] = phi0
    c.field("phi")[:] = phi0
    out["A"], out["b"] = c.assemble()
    c.field("phi")[:] = 0.0
    for _ in range(3):
        c.step()
    out["phi_it3"] = c.field("phi").copy()
    return out


if __name__ == "__main__":
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import pyoracle

    np.savez_compressed(OUT, **generate(pyoracle))
    print(OUT, os.path.getsize(OUT))
    np.savez_compressed(OUT_COND, **generate_conduction(pyoracle))
    print(OUT_COND, os.path.getsize(OUT_COND))
