"""Oracle (test infrastructure only): ctypes view of oracle/_build/liboracle.so.

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg, always as the checker. The product (``openaccel_b200``) never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class Settings(C.Structure):
    _fields_ = [
        ("rho", C.c_double),
        ("mu", C.c_double),
        ("urf_u", C.c_double),
        ("urf_p", C.c_double),
        ("dt", C.c_double),
        ("grad_urf", C.c_double),
        ("mdot_urf", C.c_double),
        ("wall_rhs_relax", C.c_double),
        ("u_shifted", C.c_int),
        ("u_grad_shifted", C.c_int),
        ("p_shifted", C.c_int),
        ("p_grad_shifted", C.c_int),
        ("ref_node", C.c_int),
        ("mom_maxit", C.c_int),
        ("mom_rtol", C.c_double),
        ("pc_maxit", C.c_int),
        ("pc_rtol", C.c_double),
        ("hr", C.c_int),
        ("beta_max", C.c_double),
        ("du_mode", C.c_int),
    ]


class IterStats(C.Structure):
    _fields_ = [
        ("mom_iters", C.c_int * 1),
        ("mom_res", C.c_double),
        ("pc_iters", C.c_int),
        ("pc_res", C.c_double),
        ("continuity_rms", C.c_double),
        ("continuity_raw", C.c_double),
    ]


def default_settings(**kw) -> Settings:
    """Cavity-example settings (examples/cavity/input.i:46-53) with
    linear_linear velocity interpolation and the controls.h defaults."""
    d = dict(rho=1.0, mu=0.01, urf_u=0.9, urf_p=0.1, dt=1.0, grad_urf=0.5625, mdot_urf=1.0,
             wall_rhs_relax=0.75, u_shifted=1, u_grad_shifted=1, p_shifted=1, p_grad_shifted=1,
             ref_node=0, mom_maxit=200, mom_rtol=1e-12, pc_maxit=5000, pc_rtol=1e-12, hr=0, beta_max=1.0, du_mode=0)
    d.update(kw)
    return Settings(**d)


class DiffSettings(C.Structure):
    _fields_ = [
        ("shifted", C.c_int),
        ("urf", C.c_double),
        ("wall_rhs_relax", C.c_double),
        ("lower_clip", C.c_double),
        ("maxit", C.c_int),
        ("rtol", C.c_double),
    ]


def default_diff_settings(**kw) -> DiffSettings:
    """Solid energy-equation defaults: linear_linear interpolation
    (controls.h:95), energy relaxation 1 (controls.h:73), wall rhs relaxation
    0.75 (thermalEnergyAssembler.h:42), clip at 0, CG to 1e-10."""
    d = dict(shifted=1, urf=1.0, wall_rhs_relax=0.75, lower_clip=0.0, maxit=20000, rtol=1e-10)
    d.update(kw)
    return DiffSettings(**d)


class SstConstants(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("sigma_k1", "sigma_k2", "sigma_w1", "sigma_w2", "beta1", "beta2",
                                           "gamma1", "gamma2", "a1", "beta_star", "prod_limit", "cmu")]


SST_IN = ("k", "omega", "k_prev", "rho", "mu", "ymin", "gradU", "gradK", "gradW", "div", "vol", "mut_old",
          "pk_wall")
SST_OUT = ("mut", "F1", "Pk", "k_diag", "k_rhs", "w_diag", "w_rhs")


class SstIn(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in SST_IN] + [("wall_node", C.POINTER(C.c_int))]


class SstOut(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in SST_OUT]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER
        dp, ip = P(C.c_double), P(C.c_int)
        L.orc_case_create.restype = C.c_void_p
        L.orc_case_create.argtypes = [C.c_int, C.c_int, dp, ip, C.c_int, ip, ip, ip, C.c_int, dp,
                                      P(Settings)]
        L.orc_case_destroy.argtypes = [C.c_void_p]
        L.orc_set_ref_nodes.argtypes = [C.c_void_p, ip, C.c_int]
        L.orc_set_boundary_types.argtypes = [C.c_void_p, ip, C.c_int, C.c_int]
        L.orc_set_boundary_types.restype = C.c_int
        L.orc_case_field.restype = dp
        L.orc_case_field.argtypes = [C.c_void_p, C.c_char_p, P(C.c_long)]
        L.orc_case_nnz.restype = C.c_int
        L.orc_case_nnz.argtypes = [C.c_void_p]
        L.orc_case_mass_scale.restype = C.c_double
        L.orc_case_mass_scale.argtypes = [C.c_void_p]
        L.orc_apply_coeff.restype = None
        L.orc_apply_coeff.argtypes = [C.c_void_p, C.c_int, P(C.c_double), P(C.c_double), P(C.c_int), C.c_int,
                                      P(C.c_double), P(C.c_double)]
        L.orc_advance_time.restype = None
        L.orc_advance_time.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_set_solver.restype = None
        L.orc_set_solver.argtypes = [C.c_void_p, C.c_int]
        L.orc_gmres_ilu.restype = C.c_int
        L.orc_gmres_ilu.argtypes = [C.c_void_p, C.c_int, P(C.c_double), P(C.c_double), P(C.c_double), C.c_double,
                                    C.c_int, C.c_int, P(C.c_double)]
        L.orc_case_graph.argtypes = [C.c_void_p, ip, ip]
        for name in ["orc_initialize", "orc_update_mdot", "orc_update_div", "orc_update_grad_p",
                     "orc_update_grad_u", "orc_update_blending_u"]:
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_assemble_momentum.argtypes = [C.c_void_p, dp, dp]
        L.orc_assemble_pcorr.argtypes = [C.c_void_p, dp, dp]
        L.orc_assemble_scalar_transport.restype = None
        L.orc_assemble_scalar_transport.argtypes = [C.c_void_p, dp, dp, dp, dp, C.c_double, dp, dp]
        L.orc_bicgstab.restype = C.c_int
        L.orc_bicgstab.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, C.c_double, C.c_int, dp]
        L.orc_simple_iteration.argtypes = [C.c_void_p, P(IterStats)]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_hex8_scs_areav.argtypes = [dp, dp]
        L.orc_hex8_scv_volumes.argtypes = [dp, dp]
        L.orc_hex8_scv_volumes.restype = C.c_int
        L.orc_hex8_grad_op.argtypes = [dp, dp, C.c_int]
        L.orc_hex8_grad_op.restype = C.c_int
        L.orc_hex8_shape.argtypes = [dp, C.c_int]
        L.orc_get_threads.restype = C.c_int
        L.orc_tet4_scs_areav.argtypes = [dp, dp]
        L.orc_tet4_scv_volumes.argtypes = [dp, dp]
        L.orc_tet4_scv_volumes.restype = C.c_int
        L.orc_tet4_grad_op.argtypes = [dp, dp]
        L.orc_tet4_grad_op.restype = C.c_int
        L.orc_tet4_shape.argtypes = [dp, C.c_int]
        L.orc_tri3_face_areav.argtypes = [dp, dp]
        L.orc_diff_create.restype = C.c_void_p
        L.orc_diff_create.argtypes = [C.c_int, C.c_int, dp, ip, C.c_int, ip, ip, ip, C.c_int, ip, dp,
                                      P(DiffSettings)]
        L.orc_diff_destroy.argtypes = [C.c_void_p]
        L.orc_diff_field.restype = dp
        L.orc_diff_field.argtypes = [C.c_void_p, C.c_char_p, P(C.c_long)]
        L.orc_diff_nnz.restype = C.c_int
        L.orc_diff_nnz.argtypes = [C.c_void_p]
        L.orc_diff_graph.argtypes = [C.c_void_p, ip, ip]
        L.orc_diff_assemble.argtypes = [C.c_void_p, dp, dp]
        L.orc_diff_cg.restype = C.c_int
        L.orc_diff_cg.argtypes = [C.c_void_p, dp, dp, dp, C.c_double, C.c_int, dp]
        L.orc_diff_spmv.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_diff_bicgstab.restype = C.c_int
        L.orc_diff_bicgstab.argtypes = [C.c_void_p, dp, dp, dp, C.c_double, C.c_int, dp]
        L.orc_sst_default_constants.argtypes = [P(SstConstants)]
        L.orc_sst_nodes.argtypes = [C.c_int, P(SstConstants), C.c_double, C.c_double, P(SstIn), P(SstOut)]
        L.orc_sst_diffusivities.argtypes = [C.c_int, P(SstConstants)] + [dp] * 6
        L.orc_diff_step.restype = C.c_int
        L.orc_diff_step.argtypes = [C.c_void_p, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


class FlowCase:
    """Oracle flow case over a ``meshgen.HexMesh``."""

    def __init__(self, mesh, settings: Settings | None = None, U0=None):
        self.mesh = mesh
        self.settings = settings or default_settings()
        self._keep = [np.ascontiguousarray(mesh.coords, np.float64),
                      np.ascontiguousarray(mesh.conn, np.int32),
                      np.ascontiguousarray(mesh.face_elem, np.int32),
                      np.ascontiguousarray(mesh.face_ord, np.int32),
                      np.ascontiguousarray(mesh.face_bnd, np.int32),
                      np.ascontiguousarray(mesh.bnd_velocity, np.float64)]
        x, conn, fe, fo, fb, bv = self._keep
        self.h = lib().orc_case_create(mesh.nn, mesh.ne, _dp(x), _ip(conn), mesh.nf, _ip(fe), _ip(fo),
                                       _ip(fb), bv.shape[0], _dp(bv), C.byref(self.settings))
        self.nnz = lib().orc_case_nnz(self.h)
        if U0 is not None:
            self.field("U")[:] = np.asarray(U0, np.float64).ravel()

    def close(self):
        if self.h:
            lib().orc_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, name: str) -> np.ndarray:
        n = C.c_long(0)
        p = lib().orc_case_field(self.h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,))

    def graph(self):
        rp = np.zeros(self.mesh.nn + 1, np.int32)
        cols = np.zeros(self.nnz, np.int32)
        lib().orc_case_graph(self.h, _ip(rp), _ip(cols))
        return rp, cols

    def set_ref_nodes(self, nodes):
        n = np.ascontiguousarray(nodes, np.int32)
        self._keep.append(n)
        lib().orc_set_ref_nodes(self.h, _ip(n), int(n.size))

    def set_boundary_types(self, types, correct_gradients=False):
        """Boundary physical types by boundary index: 0 no-slip wall, 1 symmetry."""
        t = np.ascontiguousarray(types, np.int32)
        if lib().orc_set_boundary_types(self.h, _ip(t), int(t.size), int(bool(correct_gradients))) != 0:
            raise ValueError("orc_set_boundary_types: one type per boundary, 0 or 1")

    def initialize(self):
        lib().orc_initialize(self.h)

    def assemble_momentum(self):
        A = np.zeros(9 * self.nnz)
        b = np.zeros(3 * self.mesh.nn)
        lib().orc_assemble_momentum(self.h, _dp(A), _dp(b))
        return A, b

    def assemble_pcorr(self):
        A = np.zeros(self.nnz)
        b = np.zeros(self.mesh.nn)
        lib().orc_assemble_pcorr(self.h, _dp(A), _dp(b))
        return A, b

    def assemble_transport(self, phi, gamma, src_diag, src_rhs, urf):
        """k / omega transport system of a nodal field phi with nodal diffusivity
        gamma, per-node source terms and diagonal relaxation 1/urf."""
        arrs = [np.ascontiguousarray(a, np.float64) for a in (phi, gamma, src_diag, src_rhs)]
        A = np.zeros(self.nnz)
        b = np.zeros(self.mesh.nn)
        lib().orc_assemble_scalar_transport(self.h, *[_dp(a) for a in arrs], float(urf), _dp(A), _dp(b))
        return A, b

    def update_mdot(self):
        lib().orc_update_mdot(self.h)

    def update_div(self):
        lib().orc_update_div(self.h)

    def update_grad_p(self):
        lib().orc_update_grad_p(self.h)

    def update_grad_u(self):
        lib().orc_update_grad_u(self.h)

    def update_blending_u(self):
        lib().orc_update_blending_u(self.h)

    def bicgstab(self, bs, A, b, rtol=1e-12, maxit=2000):
        x = np.zeros_like(b)
        res = C.c_double(0)
        it = lib().orc_bicgstab(self.h, bs, _dp(A), _dp(b), _dp(x), rtol, maxit, C.byref(res))
        return x, it, res.value

    def simple_iteration(self):
        st = IterStats()
        lib().orc_simple_iteration(self.h, C.byref(st))
        return dict(mom_iters=st.mom_iters[0], mom_res=st.mom_res, pc_iters=st.pc_iters,
                    pc_res=st.pc_res, continuity_rms=st.continuity_rms, continuity_raw=st.continuity_raw)

    def apply_coeff(self, bs, A, b, nodes, rhs, lhs):
        """The oracle's applyCoeff_ restatement: adds an element system into A, b in place."""
        nodes = np.ascontiguousarray(nodes, np.int32)
        lib().orc_apply_coeff(self.h, bs, _dp(A), _dp(b), nodes.ctypes.data_as(C.POINTER(C.c_int)), int(nodes.size),
                              _dp(np.ascontiguousarray(rhs, np.float64)), _dp(np.ascontiguousarray(lhs, np.float64)))

    def advance_time(self, scheme, dt):
        """Start a time step: scheme 1 BDF1, 2 BDF2."""
        lib().orc_advance_time(self.h, scheme, dt)

    def set_solver(self, kind):
        """0: Jacobi-BiCGStab (parity reference); 1 or "reference": the cavity
        example's GMRES + block-Jacobi ILU(0) configuration."""
        lib().orc_set_solver(self.h, {"reference": 1, "ilu-bicgstab": 2}.get(kind, kind))

    def gmres_ilu(self, bs, A, b, rtol=1e-12, maxit=2000, restart=50):
        x = np.zeros_like(b)
        res = C.c_double(0)
        it = lib().orc_gmres_ilu(self.h, bs, _dp(A), _dp(b), _dp(x), rtol, maxit, restart, C.byref(res))
        return x, it, res.value

    def mass_scale(self):
        """Continuity-residual scale rho U_ref h^2 of the case."""
        return lib().orc_case_mass_scale(self.h)


def hex8_scs_areav(x):
    x = np.ascontiguousarray(x, np.float64).reshape(8, 3)
    a = np.zeros((12, 3))
    lib().orc_hex8_scs_areav(_dp(x), _dp(a))
    return a


def hex8_scv_volumes(x):
    x = np.ascontiguousarray(x, np.float64).reshape(8, 3)
    v = np.zeros(8)
    lib().orc_hex8_scv_volumes(_dp(x), _dp(v))
    return v


def hex8_grad_op(x, shifted=True):
    x = np.ascontiguousarray(x, np.float64).reshape(8, 3)
    g = np.zeros((12, 8, 3))
    err = lib().orc_hex8_grad_op(_dp(x), _dp(g), int(shifted))
    return g, err


def hex8_shape(shifted=True):
    N = np.zeros((12, 8))
    lib().orc_hex8_shape(_dp(N), int(shifted))
    return N


class DiffCase:
    """Oracle tet4 scalar-diffusion case over a ``meshgen.TetMesh``."""

    def __init__(self, mesh, gamma=None, src=None, settings: DiffSettings | None = None):
        self.mesh = mesh
        self.settings = settings or default_diff_settings()
        self._keep = [np.ascontiguousarray(mesh.coords, np.float64),
                      np.ascontiguousarray(mesh.conn, np.int32),
                      np.ascontiguousarray(mesh.face_elem, np.int32),
                      np.ascontiguousarray(mesh.face_ord, np.int32),
                      np.ascontiguousarray(mesh.face_bnd, np.int32),
                      np.ascontiguousarray(mesh.bnd_kind, np.int32),
                      np.ascontiguousarray(mesh.bnd_value, np.float64)]
        x, conn, fe, fo, fb, bk, bv = self._keep
        self.h = lib().orc_diff_create(mesh.nn, mesh.ne, _dp(x), _ip(conn), mesh.nf, _ip(fe), _ip(fo), _ip(fb),
                                       bk.shape[0], _ip(bk), _dp(bv), C.byref(self.settings))
        self.nnz = lib().orc_diff_nnz(self.h)
        if gamma is not None:
            self.field("gamma")[:] = gamma
        if src is not None:
            self.field("src")[:] = src

    def close(self):
        if self.h:
            lib().orc_diff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, name: str) -> np.ndarray:
        n = C.c_long(0)
        p = lib().orc_diff_field(self.h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,))

    def graph(self):
        rp = np.zeros(self.mesh.nn + 1, np.int32)
        cols = np.zeros(self.nnz, np.int32)
        lib().orc_diff_graph(self.h, _ip(rp), _ip(cols))
        return rp, cols

    def assemble(self):
        A = np.zeros(self.nnz)
        b = np.zeros(self.mesh.nn)
        lib().orc_diff_assemble(self.h, _dp(A), _dp(b))
        return A, b

    def cg(self, A, b, rtol=1e-10, maxit=20000):
        x = np.zeros_like(b)
        res = C.c_double(0)
        it = lib().orc_diff_cg(self.h, _dp(A), _dp(b), _dp(x), rtol, maxit, C.byref(res))
        return x, it, res.value

    def bicgstab(self, A, b, rtol=1e-10, maxit=20000):
        x = np.zeros_like(b)
        res = C.c_double(0)
        it = lib().orc_diff_bicgstab(self.h, _dp(A), _dp(b), _dp(x), rtol, maxit, C.byref(res))
        return x, it, res.value

    def spmv(self, A, x):
        y = np.zeros(self.mesh.nn)
        xx = np.ascontiguousarray(x, np.float64)
        lib().orc_diff_spmv(self.h, _dp(A), _dp(xx), _dp(y))
        return y

    def step(self):
        res = C.c_double(0)
        it = lib().orc_diff_step(self.h, C.byref(res))
        return it, res.value


def tet4_scs_areav(x):
    x = np.ascontiguousarray(x, np.float64).reshape(4, 3)
    a = np.zeros((6, 3))
    lib().orc_tet4_scs_areav(_dp(x), _dp(a))
    return a


def tet4_scv_volumes(x):
    x = np.ascontiguousarray(x, np.float64).reshape(4, 3)
    v = np.zeros(4)
    lib().orc_tet4_scv_volumes(_dp(x), _dp(v))
    return v


def tet4_grad_op(x):
    x = np.ascontiguousarray(x, np.float64).reshape(4, 3)
    g = np.zeros((4, 3))
    err = lib().orc_tet4_grad_op(_dp(x), _dp(g))
    return g, err


def tet4_shape(shifted=True):
    N = np.zeros((6, 4))
    lib().orc_tet4_shape(_dp(N), int(shifted))
    return N


def tri3_face_areav(p):
    p = np.ascontiguousarray(p, np.float64).reshape(3, 3)
    a = np.zeros((3, 3))
    lib().orc_tri3_face_areav(_dp(p), _dp(a))
    return a


def sst_constants() -> SstConstants:
    c = SstConstants()
    lib().orc_sst_default_constants(C.byref(c))
    return c


def sst_nodes(fields: dict, dt=1.0, mut_urf=1.0, constants: SstConstants | None = None) -> dict:
    """Node-level SST updates on numpy fields (``SST_IN`` names plus
    ``wall_node``); returns the ``SST_OUT`` arrays."""
    nn = fields["k"].shape[0]
    keep = {n: np.ascontiguousarray(fields[n], np.float64) for n in SST_IN if fields.get(n) is not None}
    wall = np.ascontiguousarray(fields["wall_node"], np.int32)
    si = SstIn(**{n: (_dp(keep[n]) if n in keep else None) for n in SST_IN}, wall_node=_ip(wall))
    outs = {n: np.zeros(nn) for n in SST_OUT}
    so = SstOut(**{n: _dp(outs[n]) for n in SST_OUT})
    c = constants or sst_constants()
    lib().orc_sst_nodes(nn, C.byref(c), dt, mut_urf, C.byref(si), C.byref(so))
    return outs


def sst_diffusivities(mu, mut, F1, constants: SstConstants | None = None):
    """(mu_eff, gamma_k, gamma_omega) of the SST driver's viscosity updates."""
    mu, mut, F1 = (np.ascontiguousarray(a, np.float64) for a in (mu, mut, F1))
    out = [np.zeros(mu.shape[0]) for _ in range(3)]
    c = constants or sst_constants()
    lib().orc_sst_diffusivities(mu.shape[0], C.byref(c), _dp(mu), _dp(mut), _dp(F1), *[_dp(a) for a in out])
    return tuple(out)
