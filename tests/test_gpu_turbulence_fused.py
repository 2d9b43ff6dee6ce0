"""Fused u/v/w/k/omega assembly (oa_flow_enable_turbulence): one launch of
the momentum kernel assembles the momentum system and the k and omega
transport systems from the same ip geometry. Parity against the oracle's
restatement of phiAssemblerElemTerms.hpp (upwind, nodal diffusivities at the
ips, zero-gradient walls) plus the node source terms and the relaxation of the
diagonal: 1e-12 in FP64, 1e-5 in the mixed form; the momentum system is the
one the plain kernel assembles."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


def setup(oracle_mod, m, prec, seed=4, **kw):
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=seed)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(precision=prec, **kw))
    gf.set_field("U", U0)
    rng = np.random.default_rng(seed)
    state = {"p": rng.normal(0, 1, m.nn), "gradP": rng.normal(0, 1, 3 * m.nn),
             "du": rng.uniform(0.1, 1.0, 3 * m.nn), "mDot": rng.normal(0, 0.01, 12 * m.ne),
             "div": rng.normal(0, 1e-3, m.nn)}
    for k, v in state.items():
        oc.field(k)[:] = v
        gf.set_field(k, v)
    turb = {"k": rng.uniform(1e-4, 1e-2, m.nn), "omega": rng.uniform(10.0, 1e3, m.nn),
            "gammaK": rng.uniform(1e-3, 2e-2, m.nn), "gammaOmega": rng.uniform(1e-3, 2e-2, m.nn),
            "srcDiagK": rng.uniform(0.0, 1e-3, m.nn), "srcRhsK": rng.normal(0, 1e-5, m.nn),
            "srcDiagOmega": rng.uniform(0.0, 1e-2, m.nn), "srcRhsOmega": rng.normal(0, 1e-2, m.nn)}
    return oc, gf, turb


@pytest.mark.parametrize("prec,mesh", [(rt.OA_PREC_FP64, "cavity"), (rt.OA_PREC_MIXED, "cavity"),
                                       (rt.OA_PREC_FP64, "star5")])
def test_fused_assembly_parity(oracle_mod, prec, mesh):
    m = meshgen.cavity(7, perturb=0.2, seed=8) if mesh == "cavity" else meshgen.star_prism(5, 4, 3, perturb=0.2)
    oc, gf, turb = setup(oracle_mod, m, prec)
    A_plain, b_plain = gf.assemble_momentum()
    urf_k, urf_w = 0.8, 0.7
    gf.enable_turbulence(urf_k, urf_w)
    for k, v in turb.items():
        gf.set_field(k, v)
    A_m, b_m = gf.assemble_momentum()
    # the momentum system is unchanged by the fusion
    np.testing.assert_array_equal(A_m, A_plain)
    np.testing.assert_array_equal(b_m, b_plain)
    A_k, b_k, A_w, b_w = gf.turbulence_systems()
    Ak_o, bk_o = oc.assemble_transport(turb["k"], turb["gammaK"], turb["srcDiagK"], turb["srcRhsK"], urf_k)
    Aw_o, bw_o = oc.assemble_transport(turb["omega"], turb["gammaOmega"], turb["srcDiagOmega"],
                                       turb["srcRhsOmega"], urf_w)
    tol = 1e-12 if prec == rt.OA_PREC_FP64 else 1e-5
    assert rel(A_k, Ak_o) < tol and rel(b_k, bk_o) < tol
    assert rel(A_w, Aw_o) < tol and rel(b_w, bw_o) < tol


def test_fused_assembly_inside_simple_iterations(oracle_mod):
    # the systems follow the flow's state: after iterations (graph mode), the
    # fused launch's k/omega systems match the oracle on the flow's mass flows
    m = meshgen.cavity(6, perturb=0.2, seed=2)
    oc, gf, turb = setup(oracle_mod, m, rt.OA_PREC_FP64)
    gf2 = rt.Flow(rt.Mesh(m), rt.default_settings(use_graphs=2))
    gf2.set_field("U", meshgen.initial_velocity(m, sigma=0.1, seed=4))
    gf2.initialize()
    gf2.enable_turbulence(0.9, 0.9)
    for k, v in turb.items():
        gf2.set_field(k, v)
    gf2.simple_iterate(3)
    A_k, b_k, _, _ = gf2.turbulence_systems()
    # the last assembly used the mass flow of the start of iteration 3; redo it
    # on the current state and compare with the oracle on the same state
    gf2.assemble_momentum()
    A_k, b_k, A_w, b_w = gf2.turbulence_systems()
    oc.field("mDot")[:] = gf2.get_field("mDot")
    Ak_o, bk_o = oc.assemble_transport(turb["k"], turb["gammaK"], turb["srcDiagK"], turb["srcRhsK"], 0.9)
    assert rel(A_k, Ak_o) < 1e-12 and rel(b_k, bk_o) < 1e-12


def test_fused_assembly_errors():
    m = meshgen.cavity(4)
    f = rt.Flow(rt.Mesh(m), rt.default_settings())
    with pytest.raises(rt.OpenAccelError) as ei:
        f.turbulence_systems()
    assert ei.value.status == 6
    with pytest.raises(rt.OpenAccelError):
        f.enable_turbulence(0.0, 0.5)
    f.enable_turbulence(0.8, 0.8)
    with pytest.raises(rt.OpenAccelError) as ei:
        f.advance_time(rt.OA_TIME_BDF1, 0.1)
    assert ei.value.status == 1
    h = rt.Flow(rt.Mesh(m), rt.default_settings(hr=1))
    with pytest.raises(rt.OpenAccelError) as ei:
        h.enable_turbulence(0.8, 0.8)
    assert ei.value.status == 1


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_turbulence_solve_and_clipped_correction(oracle_mod, prec):
    # the k and omega systems solved tightly and the corrections applied with
    # the reference's lower clip: new = old + x, or old + (SMALL - old) below it
    m = meshgen.cavity(7, perturb=0.2, seed=5)
    oc, gf, turb = setup(oracle_mod, m, prec, seed=5)
    turb["srcRhsK"] = turb["srcRhsK"] - 1e-3  # drive some k below zero
    gf.enable_turbulence(0.8, 0.7)
    for k, v in turb.items():
        gf.set_field(k, v)
    gf.assemble_momentum()
    ik, iw = gf.solve_turbulence(1e-12 if prec == rt.OA_PREC_FP64 else 1e-10, 2000)
    assert ik > 0 and iw > 0
    small = np.finfo(float).eps
    for name, g, sd, sr, urf in (("k", "gammaK", "srcDiagK", "srcRhsK", 0.8),
                                 ("omega", "gammaOmega", "srcDiagOmega", "srcRhsOmega", 0.7)):
        A, b = oc.assemble_transport(turb[name], turb[g], turb[sd], turb[sr], urf)
        x, _, res = oc.bicgstab(1, A, b, rtol=1e-13, maxit=5000)
        old = turb[name]
        new = old + x
        low = new < small
        new[low] = old[low] + (small - old[low])
        got = gf.get_field(name)
        tol = 1e-9 if prec == rt.OA_PREC_FP64 else 1e-5
        assert rel(got, new) < tol, name
        if name == "k":
            assert low.any() and np.all(got[low] == pytest.approx(small, abs=1e-18))


def test_sst_node_update_feeds_the_fused_assembly(oracle_mod):
    # the SST node kernel writes the k and omega node terms straight into the
    # flow's source fields (device pointers), reading k and omega from the
    # flow's own fields; the next fused assembly carries them
    import torch

    m = meshgen.cavity(6, perturb=0.2, seed=9)
    oc, gf, turb = setup(oracle_mod, m, rt.OA_PREC_FP64, seed=9)
    gf.enable_turbulence(0.9, 0.9)
    for k in ("k", "omega", "gammaK", "gammaOmega"):
        gf.set_field(k, turb[k])
    rng = np.random.default_rng(2)
    dev = torch.device("cuda")
    t = {"k_prev": torch.from_numpy(turb["k"]).to(dev), "rho": torch.ones(m.nn, dtype=torch.float64, device=dev),
         "mu": torch.full((m.nn,), 1e-2, dtype=torch.float64, device=dev),
         "ymin": torch.from_numpy(rng.uniform(1e-3, 0.5, m.nn)).to(dev),
         "gradU": torch.from_numpy(rng.normal(0, 1, 9 * m.nn)).to(dev),
         "gradK": torch.from_numpy(rng.normal(0, 1e-3, 3 * m.nn)).to(dev),
         "gradW": torch.from_numpy(rng.normal(0, 10, 3 * m.nn)).to(dev),
         "div": torch.zeros(m.nn, dtype=torch.float64, device=dev),
         "vol": torch.full((m.nn,), 1.0 / m.nn, dtype=torch.float64, device=dev),
         "mut_old": torch.zeros(m.nn, dtype=torch.float64, device=dev),
         "wall_node": torch.zeros(m.nn, dtype=torch.int32, device=dev)}
    for n in ("mut", "F1", "Pk"):
        t[n] = torch.empty(m.nn, dtype=torch.float64, device=dev)
    ptrs = {n: v.data_ptr() for n, v in t.items()}
    ptrs.update(k=gf.device_ptr("k"), omega=gf.device_ptr("omega"), k_diag=gf.device_ptr("srcDiagK"),
                k_rhs=gf.device_ptr("srcRhsK"), w_diag=gf.device_ptr("srcDiagOmega"),
                w_rhs=gf.device_ptr("srcRhsOmega"))
    rt.sst_node_update(m.nn, ptrs)
    torch.cuda.synchronize()
    src = {n: gf.get_field(n) for n in ("srcDiagK", "srcRhsK", "srcDiagOmega", "srcRhsOmega")}
    assert np.all(src["srcDiagK"] > 0) and np.any(src["srcRhsK"] != 0)
    gf.assemble_momentum()
    A_k, b_k, A_w, b_w = gf.turbulence_systems()
    Ak_o, bk_o = oc.assemble_transport(turb["k"], turb["gammaK"], src["srcDiagK"], src["srcRhsK"], 0.9)
    Aw_o, bw_o = oc.assemble_transport(turb["omega"], turb["gammaOmega"], src["srcDiagOmega"], src["srcRhsOmega"], 0.9)
    assert rel(A_k, Ak_o) < 1e-12 and rel(b_k, bk_o) < 1e-12
    assert rel(A_w, Aw_o) < 1e-12 and rel(b_w, bw_o) < 1e-12


@pytest.mark.parametrize("mesh", ["cavity", "star5", "symmetry"])
def test_turbulence_field_gradients(oracle_mod, mesh):
    # Green-Gauss gradients of k and omega (the SST driver's post-correction
    # gradient updates) against the oracle's scalar gradient on the same field,
    # with the turbulence fields' linear_linear operator and the relaxation;
    # on the symmetry box with the gradient correction at the symmetry nodes
    if mesh == "cavity":
        m = meshgen.cavity(7, perturb=0.2, seed=3)
    elif mesh == "star5":
        m = meshgen.star_prism(5, 4, 3, perturb=0.2)
    else:
        m = meshgen.symmetry_box(6, perturb=0.2, seed=3)
    oc, gf, turb = setup(oracle_mod, m, rt.OA_PREC_FP64, seed=3)
    with pytest.raises(rt.OpenAccelError) as ei:
        gf.update_gradient("k")
    assert ei.value.status == 6
    if mesh == "symmetry":
        types = [rt.OA_BTYPE_WALL, rt.OA_BTYPE_WALL, rt.OA_BTYPE_SYMMETRY, rt.OA_BTYPE_SYMMETRY]
        oc.set_boundary_types(types, correct_gradients=True)
        gf.set_boundary_types(types, correct_gradients=True)
    gf.enable_turbulence(0.8, 0.8)
    for name, grad in (("k", "gradK"), ("omega", "gradOmega")):
        gf.set_field(name, turb[name])
        oc.field("p")[:] = turb[name]
        oc.field("gradP")[:] = 0.0
        for _ in range(2):
            oc.update_grad_p()
            gf.update_gradient(name)
        assert rel(gf.get_field(grad), oc.field("gradP")) < 1e-12, name


def test_sst_chain_on_device(oracle_mod):
    # one SST update entirely on the device, through the library's own fields:
    # k / omega gradients (oa_update_gradient), the node update (mu_t, F1,
    # node terms written into the flow's source fields), then mu_eff and the
    # F1-blended diffusivities written into the flow's "mu", "gammaK" and
    # "gammaOmega"; each stage against the oracle on the same inputs
    import torch

    m = meshgen.cavity(6, perturb=0.2, seed=12)
    oc, gf, turb = setup(oracle_mod, m, rt.OA_PREC_FP64, seed=12)
    gf.enable_turbulence(0.9, 0.9)
    for k in ("k", "omega"):
        gf.set_field(k, turb[k])
    gf.update_gradient("k")
    gf.update_gradient("omega")
    grads = {}
    for name in ("k", "omega"):
        oc.field("p")[:] = turb[name]
        oc.field("gradP")[:] = 0.0
        oc.update_grad_p()
        grads[name] = oc.field("gradP").copy()
    assert rel(gf.get_field("gradK"), grads["k"]) < 1e-12 and rel(gf.get_field("gradOmega"), grads["omega"]) < 1e-12
    rng = np.random.default_rng(4)
    dev = torch.device("cuda")
    host = {"k_prev": turb["k"], "rho": np.ones(m.nn), "mu": np.full(m.nn, 1e-2), "ymin": rng.uniform(1e-3, 0.5, m.nn),
            "gradU": rng.normal(0, 1, 9 * m.nn), "div": np.zeros(m.nn), "vol": gf.mesh.dual_volume(),
            "mut_old": np.zeros(m.nn)}
    t = {n: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for n, v in host.items()}
    t["wall_node"] = torch.zeros(m.nn, dtype=torch.int32, device=dev)
    for n in ("mut", "F1", "Pk"):
        t[n] = torch.empty(m.nn, dtype=torch.float64, device=dev)
    ptrs = {n: v.data_ptr() for n, v in t.items()}
    ptrs.update(k=gf.device_ptr("k"), omega=gf.device_ptr("omega"), gradK=gf.device_ptr("gradK"),
                gradW=gf.device_ptr("gradOmega"), k_diag=gf.device_ptr("srcDiagK"), k_rhs=gf.device_ptr("srcRhsK"),
                w_diag=gf.device_ptr("srcDiagOmega"), w_rhs=gf.device_ptr("srcRhsOmega"))
    rt.sst_node_update(m.nn, ptrs)
    rt.sst_diffusivities(m.nn, ptrs["mu"], ptrs["mut"], ptrs["F1"], gf.device_ptr("mu"), gf.device_ptr("gammaK"),
                         gf.device_ptr("gammaOmega"))
    torch.cuda.synchronize()
    ref = oracle_mod.sst_nodes(dict(host, k=turb["k"], omega=turb["omega"], gradK=grads["k"], gradW=grads["omega"],
                                    wall_node=np.zeros(m.nn, np.int32), pk_wall=None))
    for n in ("mut", "F1"):
        assert rel(t[n].cpu().numpy(), ref[n]) < 1e-12, n
    for n, g in (("k_diag", "srcDiagK"), ("k_rhs", "srcRhsK"), ("w_diag", "srcDiagOmega"), ("w_rhs", "srcRhsOmega")):
        assert rel(gf.get_field(g), ref[n]) < 1e-12, n
    mu_eff, gk, gw = oracle_mod.sst_diffusivities(host["mu"], ref["mut"], ref["F1"])
    assert rel(gf.get_field("mu"), mu_eff) < 1e-12
    assert rel(gf.get_field("gammaK"), gk) < 1e-12 and rel(gf.get_field("gammaOmega"), gw) < 1e-12


@pytest.mark.parametrize("graphs", [1, 2])
def test_sst_iterate_driver_matches_its_steps(graphs):
    # oa_flow_sst_iterate against the same sequence made of the public calls:
    # k_prev = k, one SIMPLE iteration (fused assembly), the k / omega solves,
    # their gradients, the node update and the diffusivities; bit for bit
    import torch

    m = meshgen.channel(12, 8, 6, ratio=1.1)
    rng = np.random.default_rng(3)
    k0 = 1e-3 * np.exp(0.2 * rng.standard_normal(m.nn))
    w0 = 1e2 * np.exp(0.2 * rng.standard_normal(m.nn))
    y = m.coords[:, 1]
    dev = torch.device("cuda")
    t = {"ymin": torch.from_numpy(np.minimum(y, 1.0 - y) + 1e-3).to(dev),
         "wall": torch.from_numpy((np.isclose(y, 0.0) | np.isclose(y, 1.0)).astype(np.int32)).to(dev),
         "mu": torch.full((m.nn,), 1e-3, dtype=torch.float64, device=dev)}
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=3)
    flows = []
    for _ in range(2):
        f = rt.Flow(rt.Mesh(m), rt.default_settings(use_graphs=graphs, mu=1e-3))
        f.set_boundary_types([rt.OA_BTYPE_WALL, rt.OA_BTYPE_WALL, rt.OA_BTYPE_SYMMETRY])
        f.set_field("U", U0)
        f.initialize()
        f.enable_turbulence(0.8, 0.8)
        f.set_field("k", k0)
        f.set_field("omega", w0)
        f.set_field("gammaK", np.full(m.nn, 1e-3))
        f.set_field("gammaOmega", np.full(m.nn, 1e-3))
        flows.append(f)
    a, b = flows
    n = 3
    a.sst_iterate(n, t["ymin"].data_ptr(), t["wall"].data_ptr(), t["mu"].data_ptr(), mut_urf=0.7, rtol=1e-10)
    # the same steps by hand on the second flow
    work = {nm: torch.zeros(m.nn, dtype=torch.float64, device=dev) for nm in ("mut", "F1", "Pk", "k_prev")}
    vol = torch.from_numpy(b.mesh.dual_volume()).to(dev)
    for _ in range(n):
        torch.cuda.synchronize()
        work["k_prev"].copy_(torch.from_numpy(b.get_field("k")).to(dev))
        b.simple_iterate(1)
        b.solve_turbulence(1e-10, 500)
        b.update_gradient("k")
        b.update_gradient("omega")
        ptrs = {nm: v.data_ptr() for nm, v in work.items()}
        ptrs.update(k=b.device_ptr("k"), omega=b.device_ptr("omega"), rho=b.device_ptr("rho"),
                    mu=t["mu"].data_ptr(), ymin=t["ymin"].data_ptr(), gradU=b.device_ptr("gradU"),
                    gradK=b.device_ptr("gradK"), gradW=b.device_ptr("gradOmega"), div=b.device_ptr("div"),
                    vol=vol.data_ptr(), mut_old=work["mut"].data_ptr(),
                    wall_node=t["wall"].data_ptr(), k_diag=b.device_ptr("srcDiagK"), k_rhs=b.device_ptr("srcRhsK"),
                    w_diag=b.device_ptr("srcDiagOmega"), w_rhs=b.device_ptr("srcRhsOmega"))
        rt.sst_node_update(m.nn, ptrs, dt=rt.default_settings().dt, mut_urf=0.7, stream=b.stream_handle())
        rt.sst_diffusivities(m.nn, t["mu"].data_ptr(), work["mut"].data_ptr(), work["F1"].data_ptr(),
                             b.device_ptr("mu"), b.device_ptr("gammaK"), b.device_ptr("gammaOmega"),
                             stream=b.stream_handle())
        b.sync()
    for name in ("U", "p", "k", "omega", "mu", "gammaK", "gammaOmega", "srcRhsK", "srcRhsOmega"):
        np.testing.assert_array_equal(a.get_field(name), b.get_field(name), err_msg=name)
    np.testing.assert_array_equal(a.get_field("mut"), work["mut"].cpu().numpy())
    assert np.all(a.get_field("k") > 0) and np.all(a.get_field("omega") > 0)
    assert np.all(np.isfinite(a.get_field("U"))) and a.get_field("mut").max() > 0


def test_sst_iterate_against_the_oracle(oracle_mod):
    # two SST outer iterations of the driver against the oracle composed the
    # same way: k.prevIter = k; the k / omega systems from the node terms of the
    # previous update on the iteration's starting mass flows; the SIMPLE
    # iteration; tight k / omega solves with the lower clip; gradients; node
    # update with relaxed mu_t; mu_eff and the diffusivities
    import torch

    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000, mu=1e-3)
    m = meshgen.channel(10, 8, 6, ratio=1.1)
    types = [rt.OA_BTYPE_WALL, rt.OA_BTYPE_WALL, rt.OA_BTYPE_SYMMETRY]
    rng = np.random.default_rng(8)
    k = 1e-3 * np.exp(0.2 * rng.standard_normal(m.nn))
    w = 1e2 * np.exp(0.2 * rng.standard_normal(m.nn))
    y = m.coords[:, 1]
    ymin = np.minimum(y, 1.0 - y) + 1e-3
    wall = (np.isclose(y, 0.0) | np.isclose(y, 1.0)).astype(np.int32)
    mu_lam = np.full(m.nn, 1e-3)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=8)
    urf_k, urf_w, mut_urf, small = 0.8, 0.7, 0.7, np.finfo(float).eps

    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    oc.set_boundary_types(types)
    oc.initialize()
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    gf.set_boundary_types(types)
    gf.set_field("U", U0)
    gf.initialize()
    gf.enable_turbulence(urf_k, urf_w)
    state = {"k": k.copy(), "omega": w.copy(), "gammaK": mu_lam.copy(), "gammaOmega": mu_lam.copy(),
             "srcDiagK": np.zeros(m.nn), "srcRhsK": np.zeros(m.nn), "srcDiagOmega": np.zeros(m.nn),
             "srcRhsOmega": np.zeros(m.nn), "mut": np.zeros(m.nn)}
    for n in ("k", "omega", "gammaK", "gammaOmega"):
        gf.set_field(n, state[n])
    dev = torch.device("cuda")
    t = {"ymin": torch.from_numpy(ymin).to(dev), "wall": torch.from_numpy(wall).to(dev),
         "mu": torch.from_numpy(mu_lam).to(dev)}
    vol = oc.field("vol").copy()

    def grad(phi):
        p, gp = oc.field("p").copy(), oc.field("gradP").copy()
        oc.field("p")[:] = phi
        oc.field("gradP")[:] = 0.0
        oc.update_grad_p()
        g = oc.field("gradP").copy()
        oc.field("p")[:], oc.field("gradP")[:] = p, gp
        return g

    gk, gw = np.zeros(3 * m.nn), np.zeros(3 * m.nn)
    for _ in range(2):
        k_prev = state["k"].copy()
        Ak, bk = oc.assemble_transport(state["k"], state["gammaK"], state["srcDiagK"], state["srcRhsK"], urf_k)
        Aw, bw = oc.assemble_transport(state["omega"], state["gammaOmega"], state["srcDiagOmega"],
                                       state["srcRhsOmega"], urf_w)
        oc.simple_iteration()
        for name, A, b in (("k", Ak, bk), ("omega", Aw, bw)):
            x, _, _ = oc.bicgstab(1, A, b, rtol=1e-13, maxit=5000)
            old = state[name]
            new = old + x
            low = new < small
            new[low] = old[low] + (small - old[low])
            state[name] = new
        # the gradients relax against their previous values (grad() starts from
        # zero, so it returns the new part, g times the fresh gradient)
        g = oracle_mod.default_settings().grad_urf
        gk = (1.0 - g) * gk + grad(state["k"])
        gw = (1.0 - g) * gw + grad(state["omega"])
        out = oracle_mod.sst_nodes(dict(k=state["k"], omega=state["omega"], k_prev=k_prev, rho=np.ones(m.nn),
                                        mu=mu_lam, ymin=ymin, gradU=oc.field("gradU").copy(), gradK=gk, gradW=gw,
                                        div=oc.field("div").copy(), vol=vol, mut_old=state["mut"], pk_wall=None,
                                        wall_node=wall), dt=1.0, mut_urf=mut_urf)
        state["mut"] = out["mut"]
        state["srcDiagK"], state["srcRhsK"] = out["k_diag"], out["k_rhs"]
        state["srcDiagOmega"], state["srcRhsOmega"] = out["w_diag"], out["w_rhs"]
        mu_eff, state["gammaK"], state["gammaOmega"] = oracle_mod.sst_diffusivities(mu_lam, out["mut"], out["F1"])
        oc.field("mu")[:] = mu_eff
    gf.sst_iterate(2, t["ymin"].data_ptr(), t["wall"].data_ptr(), t["mu"].data_ptr(), mut_urf=mut_urf, rtol=1e-12,
                   maxit=5000)
    for name in ("k", "omega", "gammaK", "gammaOmega", "mut", "srcRhsK", "srcRhsOmega"):
        assert rel(gf.get_field(name), state[name]) < 1e-9, name
    assert rel(gf.get_field("mu"), oc.field("mu")) < 1e-9
    for name in ("U", "p", "mDot"):
        assert rel(gf.get_field(name), oc.field(name)) < 1e-9, name
