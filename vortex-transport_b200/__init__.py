"""vortex_transport_b200: Python mirror of the reference's stepper interface.

A thin ctypes layer over the C ABI in include/vortex_b200.h (libvortex_b200.so,
built from csrc/ for sm_100a). The names follow the reference:

    read_input_files(path)        Parameters.cpp:12-64
    Problem(params)               main.cpp:99-147 host precompute (mesh, operators, IC)
    Solver(problem)               device context replacing the CPU element loop
    rk4(solver, t_step, n)        Timestepping.cpp:85-306
    forward_euler(solver, t_step) Timestepping.cpp:39-82
    evolve_elem(solver)           Timestepping.cpp:18-36 (returns DG_time_derivative_U)

Errors: a non-physical state raises NonPhysicalState carrying the reference's
check (1 left state, 2 right state, 3 c^2), the element, face point, side and
step; the reference prints and exits instead. There is no CPU fallback: if the
library or a CUDA device is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvortex_b200.so")

VT_OK = 0
VT_ERR_NONPHYSICAL_LEFT = 1
VT_ERR_NONPHYSICAL_RIGHT = 2
VT_ERR_NONPHYSICAL_C2 = 3
VT_ERR_INVALID = -1
VT_ERR_UNSUPPORTED = -2
VT_ERR_CUDA = -3
VT_ERR_NO_MEMORY = -4

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class vt_params(ctypes.Structure):
    """Mirrors `struct parameters` (Parameters.H:5-19)."""
    _fields_ = [("p", ctypes.c_int), ("domain_x", ctypes.c_float), ("domain_y", ctypes.c_float),
                ("num_element_in_x", ctypes.c_int), ("num_element_in_y", ctypes.c_int),
                ("perturb_grid", ctypes.c_float), ("integration_order", ctypes.c_int),
                ("simulation_time", ctypes.c_float), ("number_time_steps", ctypes.c_int),
                ("time_step", ctypes.c_double), ("write_every_steps", ctypes.c_int),
                ("U_initialization_type", ctypes.c_int), ("stepping_method", ctypes.c_int)]

    def __repr__(self):
        return "vt_params(" + ", ".join(f"{k}={getattr(self, k)!r}" for k, _ in self._fields_) + ")"


class vt_vortex(ctypes.Structure):
    """Vortex constants hard-coded at Element.cpp:134-143."""
    _fields_ = [(k, ctypes.c_double) for k in
                ("rho_infty", "rc", "epsilon", "gamma", "M_infty", "p_infty", "U_infty", "V_infty",
                 "x0", "y0")]


class vt_problem_info(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("K", "p", "Np", "nfq", "nqa", "nx", "ny")]


class vt_mesh_desc(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int32), ("n_elements", ctypes.c_int32),
                ("n_line_points", ctypes.c_int32), ("element_type", _ip), ("neighbours", _ip),
                ("det_jacobian", _dp), ("inv_jacobian", _dp), ("normals", _dp),
                ("side_lengths", _dp), ("inv_mass_ref", _dp), ("stiffness_ref", _dp),
                ("line_quadrature", _dp), ("phi_plus", _dp), ("phi_minus", _dp)]


class vt_error_info(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("element", ctypes.c_int), ("point", ctypes.c_int),
                ("side", ctypes.c_int), ("step", ctypes.c_int64), ("stage", ctypes.c_int)]


class vt_device_mesh(ctypes.Structure):
    """vt_mesh_desc with the per-element arrays in device memory."""
    _fields_ = [("p", ctypes.c_int32), ("n_elements", ctypes.c_int32),
                ("n_line_points", ctypes.c_int32), ("element_type", ctypes.c_void_p),
                ("neighbours", ctypes.c_void_p), ("det_jacobian", ctypes.c_void_p),
                ("inv_jacobian", ctypes.c_void_p), ("normals", ctypes.c_void_p),
                ("side_lengths", ctypes.c_void_p), ("inv_mass_ref", _dp), ("stiffness_ref", _dp),
                ("line_quadrature", _dp), ("phi_plus", _dp), ("phi_minus", _dp)]


class vt_checkpoint_info(ctypes.Structure):
    _fields_ = [("advance_steps", ctypes.c_int64), ("forward_sweep_steps", ctypes.c_int64),
                ("stage_steps", ctypes.c_int64), ("adjoint_steps", ctypes.c_int64),
                ("optimal_advance_steps", ctypes.c_int64), ("slots_used", ctypes.c_int32),
                ("all_stages", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class VortexError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class NonPhysicalState(VortexError):
    """The reference's `Error: Non-physical state!` exits (Numericalflux.cpp:42-115)."""

    def __init__(self, status: int, message: str, info: "vt_error_info"):
        super().__init__(status, message)
        self.code = info.code
        self.element = info.element
        self.point = info.point
        self.side = info.side
        self.step = info.step
        self.stage = info.stage


_lib = None

# name: (restype, argtypes)
_SIGNATURES = {
    "vt_read_input_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(vt_params)]),
    "vt_parse_input": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(vt_params)]),
    "vt_last_message": (ctypes.c_char_p, []),
    "vt_default_vortex": (None, [ctypes.POINTER(vt_vortex)]),
    "vt_problem_create": (ctypes.c_void_p, [ctypes.POINTER(vt_params), ctypes.POINTER(vt_vortex),
                                            ctypes.POINTER(ctypes.c_int)]),
    "vt_problem_destroy": (None, [ctypes.c_void_p]),
    "vt_problem_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(vt_problem_info)]),
    "vt_problem_get_array": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p,
                                            ctypes.c_size_t]),
    "vt_problem_mesh_desc": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(vt_mesh_desc)]),
    "vt_flux_from_state": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp, _dp]),
    "vt_create": (ctypes.c_void_p, [ctypes.POINTER(vt_mesh_desc), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int)]),
    "vt_destroy": (None, [ctypes.c_void_p]),
    "vt_create_structured": (ctypes.c_void_p, [ctypes.POINTER(vt_params), ctypes.POINTER(vt_vortex), ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_int)]),
    "vt_upload_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "vt_download_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "vt_upload_state_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "vt_download_state_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "vt_step_rk4": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
    "vt_step_euler": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
    "vt_step_rk4_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
    "vt_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "vt_rhs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "vt_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(vt_error_info)]),
    "vt_get_time": (ctypes.c_double, [ctypes.c_void_p]),
    "vt_set_time": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vt_totals": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "vt_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "vt_test_bulk_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint, ctypes.c_int]),
    "vt_profile_rk4_stages": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_float)]),
    "vt_batch_create": (ctypes.c_void_p, [ctypes.POINTER(vt_mesh_desc), ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]),
    "vt_batch_destroy": (None, [ctypes.c_void_p]),
    "vt_batch_size": (ctypes.c_int, [ctypes.c_void_p]),
    "vt_batch_groups": (ctypes.c_int, [ctypes.c_void_p]),
    "vt_batch_group_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]),
    "vt_batch_upload_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "vt_batch_download_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_void_p]),
    "vt_batch_set_dt": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "vt_batch_step_rk4": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "vt_batch_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(vt_error_info)]),
    "vt_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)]),
    "vt_batch_set_mapping": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "vt_set_stage_mapping": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "vt_get_stage_mapping": (ctypes.c_int, [ctypes.c_void_p]),
    "vt_batch_set_blocks_per_sm": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "vt_batch_time_groups": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    "vt_checkpoint_plan": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "vt_save_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "vt_project_vortex": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.POINTER(vt_vortex), ctypes.c_double,
                                         ctypes.c_int, _dp]),
    "vt_load_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "vt_write_state_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]),
    "vt_state_file_info": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "vt_read_state_file": (ctypes.c_int, [ctypes.c_char_p, _dp]),
    "vt_l2_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_void_p, ctypes.c_int, _dp]),
    "vt_problem_exact_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _dp]),
    "vt_adjoint_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "vt_adjoint_backward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "vt_adjoint_rk4": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p]),
    "vt_adjoint_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "vt_rhs_jvp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int]),
    "vt_rhs_vjp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int]),
    "vt_tangent_rk4": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int]),
    "vt_roe_flux": (ctypes.c_int, [_dp, _dp, ctypes.c_double, ctypes.c_double, _dp]),
    "vt_roe_flux_jvp": (ctypes.c_int, [_dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]),
    "vt_roe_flux_vjp": (None, [_dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]),
    "vt_batch_adjoint_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "vt_batch_adjoint_backward": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "vt_batch_adjoint_backward_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "vt_batch_upload_state_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "vt_batch_download_state_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "vt_batch_adjoint_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "vt_noalloc_scratch_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    "vt_step_rk4_noalloc": (ctypes.c_int, [ctypes.POINTER(vt_device_mesh), ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.POINTER(vt_error_info)]),
}


def lib() -> ctypes.CDLL:
    """The product library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise VortexError(VT_ERR_INVALID,
                              f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _message() -> str:
    m = lib().vt_last_message()
    return m.decode() if m else ""


def _check(status: int) -> None:
    if status != VT_OK:
        raise VortexError(status, _message())


def _ptr(a: np.ndarray, typ=_dp):
    return a.ctypes.data_as(typ)


# ---------------------------------------------------------------------------
# input file (Parameters.cpp:12-64)
# ---------------------------------------------------------------------------
def read_input_files(path: str) -> vt_params:
    out = vt_params()
    _check(lib().vt_read_input_file(path.encode(), ctypes.byref(out)))
    return out


def parse_input(text: str) -> vt_params:
    out = vt_params()
    _check(lib().vt_parse_input(text.encode(), ctypes.byref(out)))
    return out


def make_params(nx: int, ny: int, p: int = 3, integration_order: int = 10,
                domain_x: float = 10.0, domain_y: float = 10.0, perturb_grid: float = 0.0,
                simulation_time: float = 14.14213562373, number_time_steps: int = 10000,
                time_step: float | None = None, write_every_steps: int = 250,
                U_initialization_type: int = 0, stepping_method: int = 1) -> vt_params:
    """Parameters for a problem; defaults are input_files/input with io=10."""
    prm = vt_params()
    prm.p, prm.domain_x, prm.domain_y = p, domain_x, domain_y
    prm.num_element_in_x, prm.num_element_in_y = nx, ny
    prm.perturb_grid, prm.integration_order = perturb_grid, integration_order
    prm.simulation_time, prm.number_time_steps = simulation_time, number_time_steps
    prm.time_step = (time_step if time_step is not None
                     else float(repr(simulation_time)) / float(number_time_steps))
    prm.write_every_steps = write_every_steps
    prm.U_initialization_type, prm.stepping_method = U_initialization_type, stepping_method
    return prm


def default_vortex() -> vt_vortex:
    v = vt_vortex()
    lib().vt_default_vortex(ctypes.byref(v))
    return v


def vortex(epsilon=None, M_infty=None, x0=None, y0=None, p_infty=None, **kw) -> vt_vortex:
    """The reference vortex with some constants replaced. When M_infty changes
    and p_infty is not given, p_infty = 1 / (gamma M_infty^2) keeps the
    free stream at unit speed and Mach M_infty (20/7 at the default 0.5)."""
    v = default_vortex()
    if epsilon is not None:
        v.epsilon = epsilon
    if M_infty is not None:
        v.M_infty = M_infty
        if p_infty is None:
            v.p_infty = 1.0 / (v.gamma * M_infty * M_infty)
    if p_infty is not None:
        v.p_infty = p_infty
    if x0 is not None:
        v.x0 = x0
    if y0 is not None:
        v.y0 = y0
    for k, val in kw.items():
        setattr(v, k, val)
    return v


def flux_from_state(U: np.ndarray) -> np.ndarray:
    U = np.ascontiguousarray(U, dtype=np.float64)
    K, Np = U.shape[0], U.shape[1]
    p = {1: 0, 3: 1, 6: 2, 10: 3}[Np]
    F = np.empty((K, Np, 2, 4))
    _check(lib().vt_flux_from_state(K, p, _ptr(U), _ptr(F)))
    return F


# ---------------------------------------------------------------------------
# host precompute
# ---------------------------------------------------------------------------
def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def write_state_file(path: str, p: int, U: np.ndarray, time: float = 0.0) -> None:
    """Full-precision state file (the format of vt_save_state); no GPU needed."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    _check(lib().vt_write_state_file(os.fsencode(path), int(p), U.shape[0], float(time), _ptr(U)))


def read_state_file(path: str):
    """(U, p, time) from a state file; no GPU needed."""
    p, K, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    _check(lib().vt_state_file_info(os.fsencode(path), ctypes.byref(p), ctypes.byref(K), ctypes.byref(t)))
    Np = (p.value + 1) * (p.value + 2) // 2
    U = np.empty((K.value, Np, 4))
    _check(lib().vt_read_state_file(os.fsencode(path), _ptr(U)))
    return U, p.value, t.value


def checkpoint_plan(nsteps: int, nsnapshots: int) -> dict:
    """Schedule of the binomial checkpointing of an nsteps-step adjoint run
    with nsnapshots stored states (host only)."""
    info = vt_checkpoint_info()
    _check(lib().vt_checkpoint_plan(int(nsteps), int(nsnapshots), ctypes.byref(info)))
    return info.as_dict()


def _vec4(x) -> np.ndarray:
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    assert x.shape == (4,), x.shape
    return x


def roe_flux(uL, uR, n):
    """(flux, code): the Roe flux in the stage kernels' algebra, on the host."""
    f = np.empty(4)
    code = lib().vt_roe_flux(_ptr(_vec4(uL)), _ptr(_vec4(uR)), float(n[0]), float(n[1]), _ptr(f))
    return f, code


def roe_flux_jvp(uL, uR, n, duL, duR) -> np.ndarray:
    df = np.empty(4)
    lib().vt_roe_flux_jvp(_ptr(_vec4(uL)), _ptr(_vec4(uR)), float(n[0]), float(n[1]), _ptr(_vec4(duL)),
                          _ptr(_vec4(duR)), _ptr(df))
    return df


def roe_flux_vjp(uL, uR, n, bflux):
    """(buL, buR) = transposed Roe Jacobian applied to bflux."""
    buL, buR = np.zeros(4), np.zeros(4)
    lib().vt_roe_flux_vjp(_ptr(_vec4(uL)), _ptr(_vec4(uR)), float(n[0]), float(n[1]), _ptr(_vec4(bflux)),
                          _ptr(buL), _ptr(buR))
    return buL, buR


_ARRAY_SHAPES = {
    "vertices": lambda i: (i.K, 3, 2), "conn": lambda i: (i.K, 3), "type": lambda i: (i.K,),
    "nodes_ref": lambda i: (i.Np, 2), "nodes_phys": lambda i: (i.K, i.Np, 2),
    "line_quad": lambda i: (i.nfq, 2), "area_quad": lambda i: (i.nqa, 3),
    "minv_ref": lambda i: (i.Np, i.Np), "stiff_ref": lambda i: (2, i.Np, i.Np),
    "phi_plus": lambda i: (3, i.Np, i.nfq), "phi_minus": lambda i: (3, i.Np, i.nfq),
    "jac": lambda i: (i.K, 4), "jinv": lambda i: (i.K, 4), "detj": lambda i: (i.K,),
    "detjinv": lambda i: (i.K,), "normals": lambda i: (i.K, 3, 2), "sides": lambda i: (i.K, 3),
    "U0": lambda i: (i.K, i.Np, 4), "F0": lambda i: (i.K, i.Np, 2, 4),
}


class Problem:
    """Mesh, operators and initial state built on the host (main.cpp:99-131)."""

    def __init__(self, params: vt_params, ic: vt_vortex | None = None):
        st = ctypes.c_int(0)
        self.params = params
        self._h = lib().vt_problem_create(ctypes.byref(params),
                                          ctypes.byref(ic) if ic is not None else None,
                                          ctypes.byref(st))
        if not self._h:
            raise VortexError(st.value, _message())
        info = vt_problem_info()
        _check(lib().vt_problem_get_info(self._h, ctypes.byref(info)))
        self.info = info
        self.K, self.Np, self.p, self.nfq = info.K, info.Np, info.p, info.nfq

    def array(self, name: str) -> np.ndarray:
        shape = _ARRAY_SHAPES[name](self.info)
        dtype = np.int32 if name in ("conn", "type") else np.float64
        out = np.empty(shape, dtype=dtype)
        _check(lib().vt_problem_get_array(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p),
                                          out.nbytes))
        return out

    def exact_state(self, t: float) -> np.ndarray:
        """The exactly translated vortex at time t at the nodes (periodic image)."""
        out = np.empty((self.K, self.Np, 4))
        _check(lib().vt_problem_exact_state(self._h, float(t), _ptr(out)))
        return out

    def mesh_desc(self) -> vt_mesh_desc:
        d = vt_mesh_desc()
        _check(lib().vt_problem_mesh_desc(self._h, ctypes.byref(d)))
        return d

    def close(self):
        if getattr(self, "_h", None):
            lib().vt_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mesh_desc_from_arrays(p: int, etype, conn, detj, jinv, normals, sides, minv_ref, stiff_ref,
                          line_quad, phi_plus, phi_minus):
    """A vt_mesh_desc over caller-owned numpy arrays (kept alive in the return)."""
    keep = dict(
        etype=np.ascontiguousarray(etype, dtype=np.int32),
        conn=np.ascontiguousarray(conn, dtype=np.int32),
        detj=np.ascontiguousarray(detj, dtype=np.float64),
        jinv=np.ascontiguousarray(jinv, dtype=np.float64),
        normals=np.ascontiguousarray(normals, dtype=np.float64),
        sides=np.ascontiguousarray(sides, dtype=np.float64),
        minv=np.ascontiguousarray(minv_ref, dtype=np.float64),
        stiff=np.ascontiguousarray(stiff_ref, dtype=np.float64),
        line=np.ascontiguousarray(line_quad, dtype=np.float64),
        pp=np.ascontiguousarray(phi_plus, dtype=np.float64),
        pm=np.ascontiguousarray(phi_minus, dtype=np.float64),
    )
    d = vt_mesh_desc()
    d.p = p
    d.n_elements = keep["etype"].shape[0]
    d.n_line_points = keep["line"].reshape(-1, 2).shape[0]
    d.element_type = _ptr(keep["etype"], _ip)
    d.neighbours = _ptr(keep["conn"], _ip)
    d.det_jacobian = _ptr(keep["detj"])
    d.inv_jacobian = _ptr(keep["jinv"])
    d.normals = _ptr(keep["normals"])
    d.side_lengths = _ptr(keep["sides"])
    d.inv_mass_ref = _ptr(keep["minv"])
    d.stiffness_ref = _ptr(keep["stiff"])
    d.line_quadrature = _ptr(keep["line"])
    d.phi_plus = _ptr(keep["pp"])
    d.phi_minus = _ptr(keep["pm"])
    return d, keep


# ---------------------------------------------------------------------------
# device solver
# ---------------------------------------------------------------------------
class Solver:
    """One problem resident on one GPU; the stepper runs as sm_100a kernels."""

    def __init__(self, source, device: int = 0):
        if isinstance(source, Problem):
            desc, self._keep = source.mesh_desc(), source
            K, Np = source.K, source.Np
            U0 = source.array("U0")
        else:
            desc, self._keep = source
            K = desc.n_elements
            Np = (desc.p + 1) * (desc.p + 2) // 2
            U0 = None
        st = ctypes.c_int(0)
        self._h = lib().vt_create(ctypes.byref(desc), device, ctypes.byref(st))
        if not self._h:
            raise VortexError(st.value, _message())
        self.K, self.Np, self.p, self.nfq = K, Np, desc.p, desc.n_line_points
        self.device = device
        if U0 is not None:
            self.upload(U0)

    @classmethod
    def structured(cls, params: vt_params, ic: vt_vortex | None = None, device: int = 0) -> "Solver":
        """A solver whose mesh, geometry and initial state are generated on the
        device (vt_create_structured): no host precompute of per-element data."""
        self = cls.__new__(cls)
        self._keep = None
        st = ctypes.c_int(0)
        self._h = lib().vt_create_structured(ctypes.byref(params), ctypes.byref(ic) if ic is not None else None,
                                             device, ctypes.byref(st))
        if not self._h:
            raise VortexError(st.value, _message())
        self.p = params.p
        self.Np = (params.p + 1) * (params.p + 2) // 2
        self.K = 2 * params.num_element_in_x * params.num_element_in_y
        self.nfq = None
        self.device = device
        return self

    # state transfer ---------------------------------------------------------
    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.K, self.Np, 4), U.shape
        _check(lib().vt_upload_state(self._h, U.ctypes.data_as(ctypes.c_void_p)))

    def download(self, with_flux: bool = False, out: np.ndarray | None = None):
        if out is not None:
            assert out.shape == (self.K, self.Np, 4) and out.dtype == np.float64
            assert out.flags["C_CONTIGUOUS"]
        U = out if out is not None else np.empty((self.K, self.Np, 4))
        F = np.empty((self.K, self.Np, 2, 4)) if with_flux else None
        _check(lib().vt_download_state(self._h, U.ctypes.data_as(ctypes.c_void_p),
                                       F.ctypes.data_as(ctypes.c_void_p) if with_flux else None))
        return (U, F) if with_flux else U

    def upload_device(self, ptr: int) -> None:
        _check(lib().vt_upload_state_device(self._h, ctypes.c_void_p(ptr)))

    def download_device(self, ptr: int) -> None:
        _check(lib().vt_download_state_device(self._h, ctypes.c_void_p(ptr)))

    # stepping ---------------------------------------------------------------
    def _step_status(self, status: int) -> None:
        if status in (VT_ERR_NONPHYSICAL_LEFT, VT_ERR_NONPHYSICAL_RIGHT, VT_ERR_NONPHYSICAL_C2):
            info = vt_error_info()
            lib().vt_last_error(self._h, ctypes.byref(info))
            raise NonPhysicalState(status, _message(), info)
        _check(status)

    def rk4(self, dt: float, nsteps: int = 1) -> None:
        self._step_status(lib().vt_step_rk4(self._h, float(dt), int(nsteps)))

    def rk4_async(self, dt: float, nsteps: int = 1) -> None:
        self._step_status(lib().vt_step_rk4_async(self._h, float(dt), int(nsteps)))

    def synchronize(self) -> None:
        self._step_status(lib().vt_synchronize(self._h))

    def forward_euler(self, dt: float, nsteps: int = 1) -> None:
        self._step_status(lib().vt_step_euler(self._h, float(dt), int(nsteps)))

    def rhs(self) -> np.ndarray:
        out = np.empty((self.K, self.Np, 4))
        self._step_status(lib().vt_rhs(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def project_vortex(self, problem: "Problem", ic: vt_vortex | None = None, t: float = 0.0) -> None:
        """State = L2 projection of the vortex (default: the reference's) onto
        the basis, computed on the device with the problem's area rule."""
        verts = np.ascontiguousarray(problem.array("vertices"))
        aq = np.ascontiguousarray(problem.array("area_quad"))
        ic = ic if ic is not None else default_vortex()
        _check(lib().vt_project_vortex(self._h, _ptr(verts), ctypes.byref(ic), float(t), aq.shape[0], _ptr(aq)))

    def save(self, path: str) -> None:
        """Full-precision dump of the state and time (restart with load)."""
        _check(lib().vt_save_state(self._h, os.fsencode(path)))

    def load(self, path: str) -> None:
        _check(lib().vt_load_state(self._h, os.fsencode(path)))

    def l2_error(self, U_ref, area_quad) -> np.ndarray:
        """The reference script's L2 difference between the state and U_ref
        (numpy, or a CUDA torch tensor on this device) with the area rule
        area_quad (nq x 3), computed on the device."""
        aq = np.ascontiguousarray(area_quad, dtype=np.float64).reshape(-1, 3)
        ins, _outp, _out, dev, _keep = self._state_args(U_ref)
        out = np.empty(4)
        _check(lib().vt_l2_error(self._h, aq.shape[0], _ptr(aq), ins[0], dev, _ptr(out)))
        return out

    def totals(self) -> np.ndarray:
        out = np.empty(4)
        _check(lib().vt_totals(self._h, _ptr(out)))
        return out

    # derivatives ------------------------------------------------------------
    # Arrays are (K, Np, 4) float64: numpy arrays (host) or CUDA torch tensors
    # on this solver's device (passed as device pointers); results come back in
    # the same kind as the first array argument.
    def _state_args(self, *arrays):
        dev = _is_cuda_tensor(arrays[0])
        if dev:
            import torch
            torch.cuda.current_stream(arrays[0].device).synchronize()
            keep = [a.detach().to(torch.float64).contiguous() for a in arrays]
            for a in keep:
                assert tuple(a.shape) == (self.K, self.Np, 4), a.shape
            out = torch.empty_like(keep[0])
            return [ctypes.c_void_p(a.data_ptr()) for a in keep], ctypes.c_void_p(out.data_ptr()), out, 1, keep
        keep = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in arrays]
        for a in keep:
            assert a.shape == (self.K, self.Np, 4), a.shape
        out = np.empty((self.K, self.Np, 4))
        return ([a.ctypes.data_as(ctypes.c_void_p) for a in keep], out.ctypes.data_as(ctypes.c_void_p), out, 0,
                keep)

    def adjoint_forward(self, dt: float, nsteps: int, nsnapshots: int) -> None:
        """nsteps RK4 steps keeping checkpoints for adjoint_backward."""
        self._step_status(lib().vt_adjoint_forward(self._h, float(dt), int(nsteps), int(nsnapshots)))

    def adjoint_backward(self, dJdU_T):
        """dJ/dU(0) from dJ/dU(T), for the last adjoint_forward."""
        ins, outp, out, dev, _keep = self._state_args(dJdU_T)
        self._step_status(lib().vt_adjoint_backward(self._h, ins[0], outp, dev))
        return out

    def adjoint_rk4(self, dt: float, nsteps: int, nsnapshots: int, dJdU_T: np.ndarray) -> np.ndarray:
        """Both sweeps in one call (vt_adjoint_rk4) for a cotangent known before
        the run; host arrays K x Np x 4. Leaves U(T) in the solver."""
        lam = np.ascontiguousarray(dJdU_T, dtype=np.float64)
        if lam.shape != (self.K, self.Np, 4):
            raise ValueError(f"dJdU_T must have shape {(self.K, self.Np, 4)}")
        out = np.empty_like(lam)
        self._step_status(lib().vt_adjoint_rk4(self._h, float(dt), int(nsteps), int(nsnapshots),
                                               lam.ctypes.data_as(ctypes.c_void_p),
                                               out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def adjoint_info(self) -> dict:
        info = vt_checkpoint_info()
        _check(lib().vt_adjoint_info(self._h, ctypes.byref(info)))
        return info.as_dict()

    def rhs_jvp(self, U, V):
        """R'(U) V."""
        ins, outp, out, dev, _keep = self._state_args(U, V)
        _check(lib().vt_rhs_jvp(self._h, ins[0], ins[1], outp, dev))
        return out

    def rhs_vjp(self, U, W):
        """R'(U)^T W."""
        ins, outp, out, dev, _keep = self._state_args(U, W)
        _check(lib().vt_rhs_vjp(self._h, ins[0], ins[1], outp, dev))
        return out

    def tangent_rk4(self, dt: float, nsteps: int, dU0):
        """Advances the state nsteps RK4 steps and returns the propagated dU0."""
        ins, outp, out, dev, _keep = self._state_args(dU0)
        self._step_status(lib().vt_tangent_rk4(self._h, float(dt), int(nsteps), ins[0], outp, dev))
        return out

    @property
    def stage_mapping(self) -> int:
        """Warp mapping of the stage kernel: 0 component per thread, 1 pair per thread."""
        return int(lib().vt_get_stage_mapping(self._h))

    @stage_mapping.setter
    def stage_mapping(self, mapping: int) -> None:
        _check(lib().vt_set_stage_mapping(self._h, int(mapping)))

    def profile_stages(self, dt: float, reps: int) -> np.ndarray:
        ms = (ctypes.c_float * 4)()
        self._step_status(lib().vt_profile_rk4_stages(self._h, float(dt), int(reps), ms))
        return np.array(ms[:], dtype=np.float64)

    @property
    def time(self) -> float:
        return lib().vt_get_time(self._h)

    @time.setter
    def time(self, t: float) -> None:
        _check(lib().vt_set_time(self._h, float(t)))

    @property
    def stream(self) -> int:
        return lib().vt_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().vt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# batched ensemble
# ---------------------------------------------------------------------------
class Batch:
    """Independent problems advanced together (vt_batch_* in the C ABI)."""

    def __init__(self, problems, device: int = 0):
        self._problems = list(problems)
        n = len(self._problems)
        descs = (vt_mesh_desc * n)()
        for i, pb in enumerate(self._problems):
            descs[i] = pb.mesh_desc()
        st = ctypes.c_int(0)
        self._h = lib().vt_batch_create(descs, n, device, ctypes.byref(st))
        if not self._h:
            raise VortexError(st.value, _message())
        self.n = n
        self.device = device
        self.shapes = [(pb.K, pb.Np) for pb in self._problems]
        for i, pb in enumerate(self._problems):
            self.upload(i, pb.array("U0"))

    @property
    def groups(self) -> list[tuple[int, int, int]]:
        """(p, instances, elements) per group."""
        out = []
        for g in range(lib().vt_batch_groups(self._h)):
            p, ni, ne = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
            _check(lib().vt_batch_group_info(self._h, g, ctypes.byref(p), ctypes.byref(ni),
                                             ctypes.byref(ne)))
            out.append((p.value, ni.value, ne.value))
        return out

    def upload(self, i: int, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (*self.shapes[i], 4)
        _check(lib().vt_batch_upload_state(self._h, i, U.ctypes.data_as(ctypes.c_void_p)))

    def download(self, i: int) -> np.ndarray:
        U = np.empty((*self.shapes[i], 4))
        _check(lib().vt_batch_download_state(self._h, i, U.ctypes.data_as(ctypes.c_void_p), None))
        return U

    def upload_device(self, i: int, U) -> None:
        """Instance i's state from a CUDA float64 tensor (K_i, Np_i, 4) on the batch's device."""
        assert tuple(U.shape) == (*self.shapes[i], 4) and U.is_contiguous()
        import torch
        torch.cuda.current_stream(U.device).synchronize()
        _check(lib().vt_batch_upload_state_device(self._h, i, ctypes.c_void_p(U.data_ptr())))

    def download_device(self, i: int, out) -> None:
        """Instance i's state into a CUDA float64 tensor (K_i, Np_i, 4)."""
        assert tuple(out.shape) == (*self.shapes[i], 4) and out.is_contiguous()
        _check(lib().vt_batch_download_state_device(self._h, i, ctypes.c_void_p(out.data_ptr())))

    def set_dt(self, dt) -> None:
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        assert dt.shape == (self.n,)
        _check(lib().vt_batch_set_dt(self._h, _ptr(dt)))

    def _status(self, st: int) -> None:
        if st in (VT_ERR_NONPHYSICAL_LEFT, VT_ERR_NONPHYSICAL_RIGHT, VT_ERR_NONPHYSICAL_C2):
            info, inst = vt_error_info(), ctypes.c_int(-1)
            lib().vt_batch_last_error(self._h, ctypes.byref(inst), ctypes.byref(info))
            err = NonPhysicalState(st, _message(), info)
            err.instance = inst.value
            raise err
        _check(st)

    def rk4(self, nsteps: int) -> None:
        self._status(lib().vt_batch_step_rk4(self._h, int(nsteps)))

    # adjoint ----------------------------------------------------------------
    def adjoint_forward(self, nsteps: int, nsnapshots: int) -> None:
        """nsteps RK4 steps of every instance keeping checkpoints (the instances
        of a group share one time step)."""
        self._status(lib().vt_batch_adjoint_forward(self._h, int(nsteps), int(nsnapshots)))

    def adjoint_backward(self, dJdU_T) -> list:
        """dJ/dU(0) per instance from dJ/dU(T) per instance (lists of (K_i, Np_i, 4)
        numpy arrays, or CUDA tensors: then the result is CUDA tensors too)."""
        if _is_cuda_tensor(dJdU_T[0]):
            import torch
            flat = torch.cat([t.reshape(-1) for t in dJdU_T]).to(torch.float64).contiguous()
            torch.cuda.current_stream(flat.device).synchronize()
            out = torch.empty_like(flat)
            _check(lib().vt_batch_adjoint_backward_device(self._h, ctypes.c_void_p(flat.data_ptr()),
                                                          ctypes.c_void_p(out.data_ptr())))
            res, o = [], 0
            for K, Np in self.shapes:
                res.append(out[o:o + K * Np * 4].view(K, Np, 4))
                o += K * Np * 4
            return res
        flat = np.concatenate([np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in dJdU_T])
        assert flat.size == sum(K * Np * 4 for K, Np in self.shapes)
        out = np.empty_like(flat)
        _check(lib().vt_batch_adjoint_backward(self._h, _ptr(flat), _ptr(out)))
        res, o = [], 0
        for K, Np in self.shapes:
            res.append(out[o:o + K * Np * 4].reshape(K, Np, 4))
            o += K * Np * 4
        return res

    def adjoint_info(self, group: int = 0) -> dict:
        info = vt_checkpoint_info()
        _check(lib().vt_batch_adjoint_info(self._h, int(group), ctypes.byref(info)))
        return info.as_dict()

    def autotune(self, trials: int = 3, cache: str | None = None) -> list[tuple[int, int]]:
        """(resident blocks per SM, warp mapping) for each group, tuned on the
        device and cached in `cache` (a JSON file keyed by the batch's makeup
        and the GPU)."""
        import hashlib
        import json
        key = None
        ng = lib().vt_batch_groups(self._h)
        if cache:
            import torch
            props = torch.cuda.get_device_properties(self.device)
            sig = json.dumps([self.groups, props.name, props.multi_processor_count])
            key = hashlib.sha1(sig.encode()).hexdigest()
            try:
                with open(cache) as f:
                    stored = json.load(f).get(key)
            except (OSError, ValueError):
                stored = None
            if stored and all(isinstance(x, list) and len(x) == 2 for x in stored):
                bps = (ctypes.c_int * ng)(*[x[0] for x in stored])
                maps = (ctypes.c_int * ng)(*[x[1] for x in stored])
                _check(lib().vt_batch_set_mapping(self._h, maps))
                _check(lib().vt_batch_set_blocks_per_sm(self._h, bps))
                return [tuple(x) for x in stored]
        bps = (ctypes.c_int * ng)()
        maps = (ctypes.c_int * ng)()
        _check(lib().vt_batch_autotune(self._h, int(trials), bps, maps))
        best = [(int(bps[g]), int(maps[g])) for g in range(ng)]
        if cache:
            try:
                with open(cache) as f:
                    data = json.load(f)
            except (OSError, ValueError):
                data = {}
            data[key] = [list(x) for x in best]
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(data, f, indent=1)
        return best

    def time_groups(self, reps: int = 5) -> list[float]:
        """Milliseconds per RK4 step of each group run on its own (device time)."""
        ng = lib().vt_batch_groups(self._h)
        arr = (ctypes.c_float * ng)()
        _check(lib().vt_batch_time_groups(self._h, int(reps), arr))
        return [float(x) for x in arr]

    def close(self):
        if getattr(self, "_h", None):
            lib().vt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# the reference's free functions (Timestepping.H:8-9, Timestepping.cpp:18)
# ---------------------------------------------------------------------------
def rk4(solver: Solver, t_step: float, n_steps: int = 1) -> None:
    solver.rk4(t_step, n_steps)


def forward_euler(solver: Solver, t_step: float, n_steps: int = 1) -> None:
    solver.forward_euler(t_step, n_steps)


def evolve_elem(solver: Solver) -> np.ndarray:
    return solver.rhs()
