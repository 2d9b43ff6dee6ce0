"""GPU parity of the fused k-omega SST node kernel (turbulent viscosity, F1,
production, k / omega node terms) against the oracle, through the C-ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    from openaccel_b200 import runtime

    runtime.lib()
    return runtime, torch


def _fields(nn, seed, wall_frac=0.1):
    rng = np.random.default_rng(seed)
    f = dict(
        k=10 ** rng.uniform(-6, -1, nn), omega=10 ** rng.uniform(0, 5, nn), rho=rng.uniform(0.9, 1.1, nn),
        mu=np.full(nn, 1e-5), ymin=10 ** rng.uniform(-5, np.log10(0.5), nn), gradU=rng.normal(0, 100, 9 * nn),
        gradK=rng.normal(0, 1e-2, 3 * nn), gradW=rng.normal(0, 1e3, 3 * nn), div=rng.normal(0, 1e-3, nn),
        vol=rng.uniform(1e-7, 2e-7, nn), mut_old=10 ** rng.uniform(-6, -3, nn),
        wall_node=(rng.uniform(size=nn) < wall_frac).astype(np.int32), pk_wall=rng.uniform(0, 1, nn))
    f["k_prev"] = f["k"] * rng.uniform(0.9, 1.1, nn)
    return f


def _run_gpu(rt, torch, f, dt, urf, inplace=False, with_pk_wall=True):
    nn = f["k"].shape[0]
    dev = {}
    for n in rt.SST_INPUTS:
        if n == "pk_wall" and not with_pk_wall:
            continue
        dev[n] = torch.from_numpy(np.ascontiguousarray(f[n])).cuda()
    dev["wall_node"] = torch.from_numpy(f["wall_node"]).cuda()
    for n in rt.SST_OUTPUTS:
        dev[n] = torch.empty(nn, dtype=torch.float64, device="cuda")
    if inplace:
        dev["mut"] = dev["mut_old"]
    ptrs = {n: t.data_ptr() for n, t in dev.items()}
    rt.sst_node_update(nn, ptrs, dt=dt, mut_urf=urf, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return {n: dev[n].cpu().numpy() for n in rt.SST_OUTPUTS}


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("dt,urf", [(1.0, 1.0), (1e-3, 0.7)])
def test_sst_node_kernel_matches_oracle(env, oracle_mod, dt, urf):
    rt, torch = env
    f = _fields(50_000, seed=5)
    g = _run_gpu(rt, torch, f, dt, urf)
    o = oracle_mod.sst_nodes(f, dt=dt, mut_urf=urf)
    for n in rt.SST_OUTPUTS:
        assert _rel(g[n], o[n]) <= 1e-12, n


def test_sst_node_kernel_inplace_mut_and_no_wall_production(env, oracle_mod):
    rt, torch = env
    f = _fields(20_000, seed=6)
    g = _run_gpu(rt, torch, f, 1.0, 0.5, inplace=True, with_pk_wall=False)
    f2 = dict(f)
    f2["pk_wall"] = None
    o = oracle_mod.sst_nodes(f2, dt=1.0, mut_urf=0.5)
    for n in rt.SST_OUTPUTS:
        assert _rel(g[n], o[n]) <= 1e-12, n
    assert np.all(g["Pk"][f["wall_node"] == 1] == 0.0)


def test_sst_null_field_rejected(env):
    rt, _ = env
    with pytest.raises(rt.OpenAccelError):
        rt.sst_node_update(10, {"k": 0})
