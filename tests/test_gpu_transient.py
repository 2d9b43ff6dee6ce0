"""Transient runs on the GPU against the oracle: BDF1 and BDF2 (variable
step) momentum node terms (navierStokesAssemblerNodeTerms.cpp:151-427) and
the transient part of the mass divergence (flowModel.cpp:13556-13700), three
time steps of three coefficient iterations each (simulation::runTransient,
simulation.cpp:222-312), tight inner solves.

Bars: the momentum system of a transient step within 1e-12 (FP64), fields
within 1e-10 after the run."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


@pytest.mark.parametrize("scheme", [1, 2])
def test_transient_steps(oracle_mod, scheme):
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13, urf_u=1.0, urf_p=0.5)
    m = meshgen.cavity(6, perturb=0.2, seed=23)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=23)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    gf.set_field("U", U0)
    oc.initialize()
    gf.initialize()
    for step, dt in enumerate((0.1, 0.1, 0.05)):
        oc.advance_time(scheme, dt)
        gf.advance_time(scheme, dt)
        if step == 2:
            A_o, b_o = oc.assemble_momentum()
            A_g, b_g = gf.assemble_momentum()
            assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12
            assert rel(gf.get_field("Uoldold"), oc.field("U")) > 0  # three distinct levels in play
        for _ in range(3):
            oc.simple_iteration()
        gf.simple_iterate(3)
    for k in ("U", "p", "mDot", "div"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
