"""ctypes binding of the C-ABI in ``include/openaccel_b200.h``.

There is no CPU fallback: if ``_lib/libopenaccel_b200.so`` is missing or cannot
be loaded, every entry point raises. ``OpenAccelError`` carries the library's
status code and ``oa_last_error()`` message, the counterpart of the reference's
``errorMsg`` -> ``std::runtime_error`` convention (src/basic/macros.cpp:21-24).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libopenaccel_b200.so")

OA_TOPO_HEX8 = 8
OA_TOPO_TET4 = 4
OA_PREC_FP64 = 0
OA_PREC_MIXED = 1
OA_BTYPE_WALL = 0
OA_BTYPE_SYMMETRY = 1
OA_TIME_BDF1 = 1
OA_TIME_BDF2 = 2
OA_STATIC_SOLVE_MAX_ROWS = 131072

# every symbol the header declares; checked by tests on CPU
EXPORTS = [
    "oa_last_error", "oa_version", "oa_mesh_create", "oa_mesh_destroy", "oa_mesh_nnz", "oa_mesh_graph",
    "oa_mesh_dual_volume", "oa_flow_create", "oa_flow_destroy", "oa_flow_set_field", "oa_flow_get_field",
    "oa_flow_field_device_ptr", "oa_flow_set_reference_nodes", "oa_flow_set_boundary_types", "oa_flow_initialize", "oa_assemble_momentum", "oa_assemble_pcorr",
    "oa_update_mdot", "oa_update_div", "oa_update_gradient", "oa_solve", "oa_simple_iterate", "oa_flow_sync",
    "oa_flow_stream", "oa_launch_count", "oa_time_kernel", "oa_pcorr_solve_static",
    "oa_diffusion_create", "oa_diffusion_destroy", "oa_diffusion_set_field", "oa_diffusion_get_field",
    "oa_diffusion_field_device_ptr", "oa_diffusion_assemble", "oa_diffusion_solve", "oa_diffusion_step",
    "oa_diffusion_stream", "oa_diffusion_time_assembly", "oa_sst_default_constants", "oa_sst_node_update", "oa_sst_diffusivities",
    "oa_flow_last_control", "oa_flow_scales", "oa_flow_advance_time", "oa_flow_autotune", "oa_flow_set_tuning",
    "oa_flow_enable_turbulence", "oa_flow_turbulence_systems", "oa_flow_solve_turbulence", "oa_flow_sst_iterate",
]

OA_BND_FIXED_VALUE = 0
OA_BND_ZERO_FLUX = 1


class OpenAccelError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"openaccel_b200 status {status}: {msg}")
        self.status = status


class FlowSettings(C.Structure):
    _fields_ = [
        ("rho", C.c_double), ("mu", C.c_double), ("urf_u", C.c_double), ("urf_p", C.c_double),
        ("dt", C.c_double), ("grad_urf", C.c_double), ("mdot_urf", C.c_double),
        ("wall_rhs_relax", C.c_double), ("u_shifted", C.c_int), ("u_grad_shifted", C.c_int),
        ("p_shifted", C.c_int), ("p_grad_shifted", C.c_int), ("ref_node", C.c_int),
        ("mom_maxit", C.c_int), ("mom_rtol", C.c_double), ("pc_maxit", C.c_int), ("pc_rtol", C.c_double),
        ("precision", C.c_int), ("pc_amg", C.c_int), ("use_graphs", C.c_int), ("hr", C.c_int),
        ("beta_max", C.c_double), ("du_mode", C.c_int),
    ]


PHASES = ("ms_momentum_assembly", "ms_momentum_solve", "ms_pcorr_assembly", "ms_pcorr_solve", "ms_corrections")


class ControlData(C.Structure):
    """oa_control_data: the ControlData of one linear solve
    (src/equation/linearSystem.h:473-488)."""
    _fields_ = [
        ("n_iterations", C.c_int), ("fallback", C.c_int), ("solver_initial_res", C.c_double * 3),
        ("solver_final_res", C.c_double * 3), ("scaled_initial_res", C.c_double * 3),
    ]

    def as_dict(self):
        return dict(n_iterations=self.n_iterations, fallback=self.fallback,
                    solver_initial_res=list(self.solver_initial_res), solver_final_res=list(self.solver_final_res),
                    scaled_initial_res=list(self.scaled_initial_res))


class ResidualHistory:
    """Per-outer-iteration convergence record, the counterpart of the
    reference's convergence report (linearSystem::convergenceReport_,
    src/equation/linearSystem.h:464-571: per equation and component the
    solver's initial and final residuals, the scaled initial residual and the
    iteration count), kept in memory and, with ``path``, appended to a CSV
    file one row per outer iteration as the iterations are reported."""

    COLUMNS = (("iteration", "continuity_rms", "continuity_rms_raw", "mom_iters", "mom_res", "mom_fallback")
               + tuple(f"mom_{q}_{c}" for q in ("initial", "final", "scaled") for c in "uvw")
               + ("pc_iters", "pc_res", "pc_refinements", "pc_fallback", "pc_initial", "pc_final", "pc_scaled")
               + PHASES)

    def __init__(self, path=None):
        self.rows = []
        self.path = path
        if path is not None:
            with open(path, "w") as fh:
                fh.write(",".join(self.COLUMNS) + "\n")

    def add(self, stats):
        """Append the dicts Flow.simple_iterate returns (one per iteration)."""
        for st in stats:
            mom, pc = st["mom"], st["pc"]
            row = [len(self.rows) + 1, st["continuity_rms"], st["continuity_rms_raw"], st["mom_iters"],
                   st["mom_res"], mom["fallback"]]
            for q in ("solver_initial_res", "solver_final_res", "scaled_initial_res"):
                row += list(mom[q])
            row += [st["pc_iters"], st["pc_res"], st["pc_refinements"], pc["fallback"], pc["solver_initial_res"][0],
                    pc["solver_final_res"][0], pc["scaled_initial_res"][0]]
            row += [st[k] for k in PHASES]
            self.rows.append(row)
            if self.path is not None:
                with open(self.path, "a") as fh:
                    fh.write(",".join(repr(v) if isinstance(v, float) else str(v) for v in row) + "\n")

    def column(self, name):
        i = self.COLUMNS.index(name)
        return [r[i] for r in self.rows]


class Tuning(C.Structure):
    """oa_tuning: launch shapes and pressure-solve schedule chosen by oa_flow_autotune."""
    _fields_ = [("block_rows", C.c_int), ("block_elements", C.c_int), ("block_assembly", C.c_int),
                ("gcr_chunk", C.c_int), ("amg_refresh", C.c_int), ("ms_per_iteration_before", C.c_double),
                ("ms_per_iteration_after", C.c_double), ("amg_cheb_degree", C.c_int),
                ("amg_prolong_damping", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class IterStats(C.Structure):
    _fields_ = [
        ("mom_iters", C.c_int), ("pc_iters", C.c_int), ("pc_refinements", C.c_int),
        ("mom_res", C.c_double), ("pc_res", C.c_double), ("continuity_rms", C.c_double),
    ] + [(n, C.c_double) for n in PHASES] + [
        ("continuity_rms_raw", C.c_double), ("mom", ControlData), ("pc", ControlData),
    ]


class DiffusionSettings(C.Structure):
    _fields_ = [
        ("shifted", C.c_int), ("urf", C.c_double), ("wall_rhs_relax", C.c_double), ("lower_clip", C.c_double),
        ("maxit", C.c_int), ("rtol", C.c_double), ("precision", C.c_int), ("amg", C.c_int),
        ("use_graphs", C.c_int),
    ]


def default_diffusion_settings(**kw) -> DiffusionSettings:
    """Solid energy-equation defaults: linear_linear interpolation
    (controls.h:95), energy relaxation 1 (controls.h:73), wall rhs relaxation
    0.75 (thermalEnergyAssembler.h:42), clip at 0, Krylov to 1e-10."""
    d = dict(shifted=1, urf=1.0, wall_rhs_relax=0.75, lower_clip=0.0, maxit=5000, rtol=1e-10,
             precision=OA_PREC_FP64, amg=1, use_graphs=0)
    d.update(kw)
    return DiffusionSettings(**d)


SST_CONSTANTS = ("sigma_k1", "sigma_k2", "sigma_w1", "sigma_w2", "beta1", "beta2", "gamma1", "gamma2", "a1",
                 "beta_star", "prod_limit", "cmu")
SST_INPUTS = ("k", "omega", "k_prev", "rho", "mu", "ymin", "gradU", "gradK", "gradW", "div", "vol", "mut_old",
              "pk_wall")
SST_OUTPUTS = ("mut", "F1", "Pk", "k_diag", "k_rhs", "w_diag", "w_rhs")


class SstConstants(C.Structure):
    _fields_ = [(n, C.c_double) for n in SST_CONSTANTS]


class SstFields(C.Structure):
    _fields_ = ([(n, C.c_void_p) for n in SST_INPUTS] + [("wall_node", C.c_void_p)] +
                [(n, C.c_void_p) for n in SST_OUTPUTS])


def default_settings(**kw) -> FlowSettings:
    """Cavity-example defaults (examples/cavity/input.i: urf 0.9 / 0.1, physical
    timescale 1, linear_linear interpolation, pressure level at node 0) and the
    controls.h defaults (gradient urf 0.5625, relaxMass 1)."""
    d = dict(rho=1.0, mu=0.01, urf_u=0.9, urf_p=0.1, dt=1.0, grad_urf=0.5625, mdot_urf=1.0,
             wall_rhs_relax=0.75, u_shifted=1, u_grad_shifted=1, p_shifted=1, p_grad_shifted=1,
             ref_node=0, mom_maxit=200, mom_rtol=1e-6, pc_maxit=5000, pc_rtol=1e-8,
             precision=OA_PREC_FP64, pc_amg=1, use_graphs=0, hr=0, beta_max=1.0, du_mode=0)
    d.update(kw)
    return FlowSettings(**d)


_lib = None


def lib():
    """Load the CUDA library (raises if it is absent: no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OpenAccelError(-1, f"CUDA library not built: {LIB_PATH} (run python -m openaccel_b200.build)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    dp, ip, vp = P(C.c_double), P(C.c_int), C.c_void_p
    sig = {
        "oa_last_error": (C.c_char_p, []),
        "oa_version": (C.c_char_p, []),
        "oa_mesh_create": (C.c_int, [dp, C.c_int, ip, C.c_int, C.c_int, ip, ip, ip, C.c_int, P(vp)]),
        "oa_mesh_destroy": (None, [vp]),
        "oa_mesh_nnz": (C.c_int, [vp, ip]),
        "oa_mesh_graph": (C.c_int, [vp, ip, ip]),
        "oa_mesh_dual_volume": (C.c_int, [vp, dp]),
        "oa_flow_create": (C.c_int, [vp, P(FlowSettings), dp, C.c_int, P(vp)]),
        "oa_flow_destroy": (None, [vp]),
        "oa_flow_set_field": (C.c_int, [vp, C.c_char_p, dp, C.c_long]),
        "oa_flow_get_field": (C.c_int, [vp, C.c_char_p, dp, C.c_long]),
        "oa_flow_field_device_ptr": (C.c_int, [vp, C.c_char_p, P(dp)]),
        "oa_flow_set_reference_nodes": (C.c_int, [vp, ip, C.c_int]),
        "oa_flow_set_boundary_types": (C.c_int, [vp, ip, C.c_int, C.c_int]),
        "oa_flow_initialize": (C.c_int, [vp]),
        "oa_assemble_momentum": (C.c_int, [vp, dp, dp]),
        "oa_assemble_pcorr": (C.c_int, [vp, dp, dp]),
        "oa_update_mdot": (C.c_int, [vp]),
        "oa_update_div": (C.c_int, [vp]),
        "oa_update_gradient": (C.c_int, [vp, C.c_int]),
        "oa_solve": (C.c_int, [vp, C.c_int, C.c_double, C.c_int, dp, ip, dp]),
        "oa_simple_iterate": (C.c_int, [vp, C.c_int, P(IterStats)]),
        "oa_flow_last_control": (C.c_int, [vp, C.c_int, P(ControlData)]),
        "oa_flow_scales": (C.c_int, [vp, dp, dp, dp]),
        "oa_flow_advance_time": (C.c_int, [vp, C.c_int, C.c_double]),
        "oa_flow_autotune": (C.c_int, [vp, C.c_int, P(Tuning)]),
        "oa_flow_set_tuning": (C.c_int, [vp, P(Tuning)]),
        "oa_flow_enable_turbulence": (C.c_int, [vp, C.c_double, C.c_double]),
        "oa_flow_turbulence_systems": (C.c_int, [vp, dp, dp, dp, dp]),
        "oa_flow_solve_turbulence": (C.c_int, [vp, C.c_double, C.c_int, ip, ip]),
        "oa_flow_sst_iterate": (C.c_int, [vp, C.c_int, P(SstConstants), vp, vp, vp, C.c_double, C.c_double,
                                          C.c_int, vp]),
        "oa_flow_sync": (C.c_int, [vp]),
        "oa_flow_stream": (C.c_int, [vp, P(vp)]),
        "oa_launch_count": (C.c_int, [P(C.c_longlong)]),
        "oa_time_kernel": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "oa_pcorr_solve_static": (C.c_int, [C.c_int, vp, vp, vp, vp, vp, vp, C.c_double, C.c_int, ip, dp, vp]),
        "oa_diffusion_create": (C.c_int, [vp, P(DiffusionSettings), ip, dp, C.c_int, P(vp)]),
        "oa_diffusion_destroy": (None, [vp]),
        "oa_diffusion_set_field": (C.c_int, [vp, C.c_char_p, dp, C.c_long]),
        "oa_diffusion_get_field": (C.c_int, [vp, C.c_char_p, dp, C.c_long]),
        "oa_diffusion_field_device_ptr": (C.c_int, [vp, C.c_char_p, P(dp)]),
        "oa_diffusion_assemble": (C.c_int, [vp, dp, dp]),
        "oa_diffusion_solve": (C.c_int, [vp, C.c_double, C.c_int, dp, ip, dp, ip]),
        "oa_diffusion_step": (C.c_int, [vp, ip, dp, ip]),
        "oa_diffusion_stream": (C.c_int, [vp, P(vp)]),
        "oa_diffusion_time_assembly": (C.c_int, [vp, C.c_int, dp]),
        "oa_sst_default_constants": (None, [P(SstConstants)]),
        "oa_sst_node_update": (C.c_int, [C.c_int, P(SstConstants), C.c_double, C.c_double, P(SstFields), vp]),
        "oa_sst_diffusivities": (C.c_int, [C.c_int, P(SstConstants), vp, vp, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def launch_count() -> int:
    n = C.c_longlong()
    _check(lib().oa_launch_count(C.byref(n)))
    return n.value


def _check(status: int):
    if status != 0:
        raise OpenAccelError(status, lib().oa_last_error().decode())


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Mesh:
    """Device mesh (oa_mesh_create) from a ``meshgen.HexMesh`` or ``meshgen.TetMesh``."""

    def __init__(self, mesh):
        self.src = mesh
        self.nn, self.ne = int(mesh.coords.shape[0]), int(mesh.conn.shape[0])
        x = np.ascontiguousarray(mesh.coords, np.float64)
        conn = np.ascontiguousarray(mesh.conn, np.int32)
        fe = np.ascontiguousarray(mesh.face_elem, np.int32)
        fo = np.ascontiguousarray(mesh.face_ord, np.int32)
        fb = np.ascontiguousarray(mesh.face_bnd, np.int32)
        h = C.c_void_p()
        self.topo = OA_TOPO_TET4 if conn.shape[1] == 4 else OA_TOPO_HEX8
        _check(lib().oa_mesh_create(_dp(x), self.nn, _ip(conn), self.ne, self.topo, _ip(fe), _ip(fo),
                                    _ip(fb), int(fe.shape[0]), C.byref(h)))
        self.h = h
        n = C.c_int()
        _check(lib().oa_mesh_nnz(self.h, C.byref(n)))
        self.nnz = n.value

    def graph(self):
        rp = np.zeros(self.nn + 1, np.int32)
        cols = np.zeros(self.nnz, np.int32)
        _check(lib().oa_mesh_graph(self.h, _ip(rp), _ip(cols)))
        return rp, cols

    def dual_volume(self):
        v = np.zeros(self.nn)
        _check(lib().oa_mesh_dual_volume(self.h, _dp(v)))
        return v

    def close(self):
        if getattr(self, "h", None):
            lib().oa_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Flow:
    """Segregated laminar flow state on the device (oa_flow_create)."""

    FIELD_SHAPES = {"U": 3, "p": 1, "gradU": 9, "gradP": 3, "du": 3, "div": 1, "sideU": 3, "rho": 1, "mu": 1,
                    "betaU": 3, "minU": 3, "maxU": 3, "duTilde": 3, "Uold": 3, "Uoldold": 3,
                    "k": 1, "omega": 1, "gammaK": 1, "gammaOmega": 1, "srcDiagK": 1, "srcRhsK": 1,
                    "srcDiagOmega": 1, "srcRhsOmega": 1, "gradK": 3, "gradOmega": 3, "mut": 1, "F1": 1, "Pk": 1}

    def __init__(self, mesh: Mesh, settings: FlowSettings | None = None):
        self.mesh = mesh
        self.settings = settings or default_settings()
        bv = np.ascontiguousarray(mesh.src.bnd_velocity, np.float64)
        h = C.c_void_p()
        _check(lib().oa_flow_create(mesh.h, C.byref(self.settings), _dp(bv), int(bv.shape[0]), C.byref(h)))
        self.h = h

    def _len(self, name):
        if name == "mDot":
            return 12 * self.mesh.ne
        return self.FIELD_SHAPES[name] * self.mesh.nn

    def set_field(self, name, values):
        v = np.ascontiguousarray(values, np.float64).ravel()
        _check(lib().oa_flow_set_field(self.h, name.encode(), _dp(v), v.size))

    def get_field(self, name):
        v = np.zeros(self._len(name))
        _check(lib().oa_flow_get_field(self.h, name.encode(), _dp(v), v.size))
        return v

    def device_ptr(self, name) -> int:
        p = C.POINTER(C.c_double)()
        _check(lib().oa_flow_field_device_ptr(self.h, name.encode(), C.byref(p)))
        return C.cast(p, C.c_void_p).value

    def set_reference_nodes(self, nodes):
        n = np.ascontiguousarray(nodes, np.int32)
        _check(lib().oa_flow_set_reference_nodes(self.h, _ip(n), int(n.size)))

    def set_boundary_types(self, types, correct_gradients=False):
        """Boundary physical types by boundary index (OA_BTYPE_WALL,
        OA_BTYPE_SYMMETRY); see oa_flow_set_boundary_types."""
        t = np.ascontiguousarray(types, np.int32)
        _check(lib().oa_flow_set_boundary_types(self.h, _ip(t), int(t.size), int(bool(correct_gradients))))

    def initialize(self):
        _check(lib().oa_flow_initialize(self.h))

    def assemble_momentum(self, copy=True):
        A = np.zeros(9 * self.mesh.nnz) if copy else None
        b = np.zeros(3 * self.mesh.nn) if copy else None
        _check(lib().oa_assemble_momentum(self.h, _dp(A), _dp(b)))
        return A, b

    def assemble_pcorr(self, copy=True):
        A = np.zeros(self.mesh.nnz) if copy else None
        b = np.zeros(self.mesh.nn) if copy else None
        _check(lib().oa_assemble_pcorr(self.h, _dp(A), _dp(b)))
        return A, b

    def update_mdot(self):
        _check(lib().oa_update_mdot(self.h))

    def update_div(self):
        _check(lib().oa_update_div(self.h))

    def update_gradient(self, which):
        _check(lib().oa_update_gradient(self.h, {"p": 0, "U": 1, "k": 2, "omega": 3}.get(which, which)))

    def solve(self, sys, rtol, maxit):
        n = 3 * self.mesh.nn if sys in (0, "momentum") else self.mesh.nn
        x = np.zeros(n)
        it, res = C.c_int(), C.c_double()
        _check(lib().oa_solve(self.h, 0 if sys in (0, "momentum") else 1, rtol, maxit, _dp(x), C.byref(it),
                              C.byref(res)))
        return x, it.value, res.value

    def simple_iterate(self, n=1, history=None):
        """n SIMPLE outer iterations; one stats dict each, also added to
        ``history`` (a ResidualHistory) when given."""
        st = (IterStats * max(n, 1))()
        _check(lib().oa_simple_iterate(self.h, n, st))
        out = [dict(mom_iters=s.mom_iters, pc_iters=s.pc_iters, pc_refinements=s.pc_refinements,
                    mom_res=s.mom_res, pc_res=s.pc_res, continuity_rms=s.continuity_rms,
                    continuity_rms_raw=s.continuity_rms_raw, mom=s.mom.as_dict(), pc=s.pc.as_dict(),
                    **{k: getattr(s, k) for k in PHASES}) for s in st[:n]]
        if history is not None:
            history.add(out)
        return out

    def advance_time(self, scheme, dt):
        """Start a time step of size dt: scheme 1 BDF1, 2 BDF2."""
        _check(lib().oa_flow_advance_time(self.h, int(scheme), float(dt)))

    def enable_turbulence(self, urf_k=1.0, urf_omega=1.0):
        """Assemble the k and omega transport systems in the momentum launch."""
        _check(lib().oa_flow_enable_turbulence(self.h, float(urf_k), float(urf_omega)))

    def turbulence_systems(self):
        """(A_k, b_k, A_omega, b_omega) of the last momentum assembly."""
        nn, nnz = self.mesh.nn, self.mesh.nnz
        out = [np.zeros(nnz), np.zeros(nn), np.zeros(nnz), np.zeros(nn)]
        _check(lib().oa_flow_turbulence_systems(self.h, *[_dp(a) for a in out]))
        return tuple(out)

    def solve_turbulence(self, rtol=1e-8, maxit=500):
        """Solve the k and omega systems of the last assembly and correct the fields."""
        ik, iw = C.c_int(), C.c_int()
        _check(lib().oa_flow_solve_turbulence(self.h, float(rtol), int(maxit), C.byref(ik), C.byref(iw)))
        return ik.value, iw.value

    def sst_iterate(self, n, ymin, wall_node, mu_lam, mut_urf=1.0, rtol=1e-8, maxit=500, constants=None):
        """n outer iterations with the SST equations (oa_flow_sst_iterate);
        ymin, wall_node, mu_lam are device pointers (ints). Returns the flow
        stats of each iteration."""
        st = (IterStats * max(n, 1))()
        c = constants or sst_constants()
        _check(lib().oa_flow_sst_iterate(self.h, int(n), C.byref(c), C.c_void_p(int(ymin)),
                                         C.c_void_p(int(wall_node)), C.c_void_p(int(mu_lam)), float(mut_urf),
                                         float(rtol), int(maxit), C.cast(st, C.c_void_p)))
        return [dict(mom_iters=s.mom_iters, pc_iters=s.pc_iters, continuity_rms=s.continuity_rms,
                     **{k: getattr(s, k) for k in PHASES}) for s in st[:n]]

    def autotune(self, iters=3):
        """Tune launch shapes and the pressure-solve schedule; the flow state is
        restored afterwards. Returns the chosen tuning as a dict."""
        t = Tuning()
        _check(lib().oa_flow_autotune(self.h, int(iters), C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = Tuning(**{k: kw[k] for k, _ in Tuning._fields_ if k in kw})
        _check(lib().oa_flow_set_tuning(self.h, C.byref(t)))

    def last_control(self, sys):
        """ControlData of the last solve of ``sys`` ("momentum"/0 or "pcorr"/1)."""
        cd = ControlData()
        _check(lib().oa_flow_last_control(self.h, 0 if sys in (0, "momentum") else 1, C.byref(cd)))
        return cd.as_dict()

    def scales(self):
        """(U_ref, mass-flux scale rho U_ref h^2, momentum-flux scale rho U_ref^2 h^2)."""
        u, m, mo = C.c_double(), C.c_double(), C.c_double()
        _check(lib().oa_flow_scales(self.h, C.byref(u), C.byref(m), C.byref(mo)))
        return u.value, m.value, mo.value

    def sync(self):
        _check(lib().oa_flow_sync(self.h))

    def stream_handle(self) -> int:
        p = C.c_void_p()
        _check(lib().oa_flow_stream(self.h, C.byref(p)))
        return p.value or 0

    def time_kernel(self, which, reps=5) -> float:
        """Mean device time (ms) of one assembly kernel, CUDA events on the flow stream."""
        ms = C.c_double()
        w = {"momentum": 0, "pcorr": 1, "mdot": 2, "gradU": 3}.get(which, which)
        _check(lib().oa_time_kernel(self.h, w, reps, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().oa_flow_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Diffusion:
    """tet4 scalar diffusion on the device (oa_diffusion_create): the solid
    energy equation of thermalEnergyEquation::solve with a per-node source."""

    FIELDS = ("phi", "gamma", "src", "sidePhi")

    def __init__(self, mesh: Mesh, settings: DiffusionSettings | None = None):
        self.mesh = mesh
        self.settings = settings or default_diffusion_settings()
        bk = np.ascontiguousarray(mesh.src.bnd_kind, np.int32)
        bv = np.ascontiguousarray(mesh.src.bnd_value, np.float64)
        h = C.c_void_p()
        _check(lib().oa_diffusion_create(mesh.h, C.byref(self.settings), _ip(bk), _dp(bv), int(bk.size),
                                         C.byref(h)))
        self.h = h

    def set_field(self, name, values):
        v = np.ascontiguousarray(values, np.float64).ravel()
        _check(lib().oa_diffusion_set_field(self.h, name.encode(), _dp(v), v.size))

    def get_field(self, name):
        v = np.zeros(self.mesh.nn)
        _check(lib().oa_diffusion_get_field(self.h, name.encode(), _dp(v), v.size))
        return v

    def device_ptr(self, name) -> int:
        p = C.POINTER(C.c_double)()
        _check(lib().oa_diffusion_field_device_ptr(self.h, name.encode(), C.byref(p)))
        return C.cast(p, C.c_void_p).value

    def assemble(self, copy=True):
        A = np.zeros(self.mesh.nnz) if copy else None
        b = np.zeros(self.mesh.nn) if copy else None
        _check(lib().oa_diffusion_assemble(self.h, _dp(A), _dp(b)))
        return A, b

    def solve(self, rtol=None, maxit=None):
        x = np.zeros(self.mesh.nn)
        it, res, nref = C.c_int(), C.c_double(), C.c_int()
        _check(lib().oa_diffusion_solve(self.h, self.settings.rtol if rtol is None else rtol,
                                        self.settings.maxit if maxit is None else maxit, _dp(x), C.byref(it),
                                        C.byref(res), C.byref(nref)))
        return x, it.value, res.value, nref.value

    def step(self):
        it, res, nref = C.c_int(), C.c_double(), C.c_int()
        _check(lib().oa_diffusion_step(self.h, C.byref(it), C.byref(res), C.byref(nref)))
        return dict(iters=it.value, res=res.value, refinements=nref.value)

    def stream_handle(self) -> int:
        p = C.c_void_p()
        _check(lib().oa_diffusion_stream(self.h, C.byref(p)))
        return p.value or 0

    def time_assembly(self, reps=5) -> float:
        ms = C.c_double()
        _check(lib().oa_diffusion_time_assembly(self.h, reps, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().oa_diffusion_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sst_constants() -> SstConstants:
    c = SstConstants()
    lib().oa_sst_default_constants(C.byref(c))
    return c


def sst_diffusivities(nn: int, mu, mut, F1, mu_eff, gamma_k, gamma_w, constants: SstConstants | None = None,
                      stream=0):
    """mu_eff = mu + mu_t and the F1-blended k / omega diffusivities on device
    pointers (ints); asynchronous on ``stream``."""
    c = constants or sst_constants()
    args = [C.c_void_p(int(p)) for p in (mu, mut, F1, mu_eff, gamma_k, gamma_w)]
    _check(lib().oa_sst_diffusivities(int(nn), C.byref(c), *args, C.c_void_p(stream or None)))


def sst_node_update(nn: int, ptrs: dict, dt=1.0, mut_urf=1.0, constants: SstConstants | None = None, stream=0):
    """Launch the fused SST node kernel on device pointers (ints) named as
    ``SST_INPUTS`` / ``wall_node`` / ``SST_OUTPUTS``; asynchronous on ``stream``."""
    f = SstFields(**{n: ptrs.get(n) for n in SST_INPUTS + ("wall_node",) + SST_OUTPUTS})
    c = constants or sst_constants()
    _check(lib().oa_sst_node_update(int(nn), C.byref(c), dt, mut_urf, C.byref(f), C.c_void_p(stream or None)))
