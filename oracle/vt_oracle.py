"""Test infrastructure: ctypes binding of the oracle (oracle/libvt_oracle.so).

The oracle is the checker, never the product: only tests/, the smoke() check
and bench.py's cpu_baseline leg load this module. It restates the reference's
right-hand side and steppers on the CPU (see dg_oracle.h for the citations).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvt_oracle.so")
HARNESS_PATH = os.path.join(HERE, "_ref", "vt_ref_harness")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class _Mesh(ctypes.Structure):
    _fields_ = [
        ("K", ctypes.c_int), ("p", ctypes.c_int), ("Np", ctypes.c_int), ("nfq", ctypes.c_int),
        ("verts", _dp), ("conn", _ip), ("type", _ip), ("minv_ref", _dp), ("stiff_ref", _dp),
        ("phi_plus", _dp), ("phi_minus", _dp), ("line_quad", _dp),
    ]


class _Err(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("element", ctypes.c_int), ("point", ctypes.c_int),
                ("side", ctypes.c_int)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "libvt_oracle.so"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.vto_rhs.argtypes = [ctypes.POINTER(_Mesh), _dp, _dp, _dp, ctypes.POINTER(_Err)]
        L.vto_rk4.argtypes = [ctypes.POINTER(_Mesh), _dp, _dp, ctypes.c_double, ctypes.c_int,
                              ctypes.POINTER(_Err)]
        L.vto_forward_euler.argtypes = L.vto_rk4.argtypes
        L.vto_flux_from_state.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.vto_numerical_flux.argtypes = [_dp, _dp, _dp, _dp]
        L.vto_geometry.argtypes = [ctypes.POINTER(_Mesh), _dp, _dp, _dp, _dp, _dp, _dp]
        L.vto_l2_state_error.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                         _dp, _dp, _dp]
        L.vto_totals.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


@dataclass
class OracleError:
    code: int
    element: int
    point: int
    side: int


class OracleMesh:
    """Inputs the reference's per-element precompute starts from."""

    def __init__(self, p: int, verts, conn, etype, minv_ref, stiff_ref, phi_plus, phi_minus,
                 line_quad):
        self.p = int(p)
        self.Np = (self.p + 1) * (self.p + 2) // 2
        self.verts = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3, 2)
        self.K = self.verts.shape[0]
        self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(self.K, 3)
        self.etype = np.ascontiguousarray(etype, dtype=np.int32).reshape(self.K)
        self.minv_ref = np.ascontiguousarray(minv_ref, dtype=np.float64).reshape(self.Np, self.Np)
        self.stiff_ref = np.ascontiguousarray(stiff_ref, dtype=np.float64).reshape(2, self.Np, self.Np)
        self.line_quad = np.ascontiguousarray(line_quad, dtype=np.float64).reshape(-1, 2)
        self.nfq = self.line_quad.shape[0]
        self.phi_plus = np.ascontiguousarray(phi_plus, dtype=np.float64).reshape(3, self.Np, self.nfq)
        self.phi_minus = np.ascontiguousarray(phi_minus, dtype=np.float64).reshape(3, self.Np, self.nfq)
        self._m = _Mesh(self.K, self.p, self.Np, self.nfq, _d(self.verts), _i(self.conn),
                        _i(self.etype), _d(self.minv_ref), _d(self.stiff_ref), _d(self.phi_plus),
                        _d(self.phi_minus), _d(self.line_quad))

    # -- hot path -------------------------------------------------------------
    def rhs(self, U, F):
        U = np.ascontiguousarray(U, dtype=np.float64)
        F = np.ascontiguousarray(F, dtype=np.float64)
        out = np.empty((self.K, self.Np, 4))
        err = _Err()
        lib().vto_rhs(ctypes.byref(self._m), _d(U), _d(F), _d(out), ctypes.byref(err))
        return out, OracleError(err.code, err.element, err.point, err.side)

    def step(self, U, F, dt: float, nsteps: int, method: int = 1):
        """method 1: rk4 (Timestepping.cpp:85-306), 0: forward_euler (:39-82)."""
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        F = np.array(F, dtype=np.float64, copy=True, order="C")
        err = _Err()
        fn = lib().vto_rk4 if method == 1 else lib().vto_forward_euler
        fn(ctypes.byref(self._m), _d(U), _d(F), float(dt), int(nsteps), ctypes.byref(err))
        return U, F, OracleError(err.code, err.element, err.point, err.side)

    def geometry(self):
        K = self.K
        jac, jinv = np.empty((K, 4)), np.empty((K, 4))
        detj, detjinv = np.empty(K), np.empty(K)
        nrm, sides = np.empty((K, 3, 2)), np.empty((K, 3))
        lib().vto_geometry(ctypes.byref(self._m), _d(jac), _d(jinv), _d(detj), _d(detjinv), _d(nrm),
                           _d(sides))
        return dict(jac=jac, jinv=jinv, detj=detj, detjinv=detjinv, normals=nrm, sides=sides)


def flux_from_state(U) -> np.ndarray:
    U = np.ascontiguousarray(U, dtype=np.float64)
    K, Np = U.shape[0], U.shape[1]
    F = np.empty((K, Np, 2, 4))
    lib().vto_flux_from_state(K, Np, _d(U), _d(F))
    return F


def numerical_flux(uL, uR, n):
    uL = np.ascontiguousarray(uL, dtype=np.float64)
    uR = np.ascontiguousarray(uR, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    out = np.empty(4)
    code = lib().vto_numerical_flux(_d(uL), _d(uR), _d(n), _d(out))
    return out, code


def l2_state_error(basis_q, area_quad, detj, Ua, Ub) -> np.ndarray:
    basis_q = np.ascontiguousarray(basis_q, dtype=np.float64)
    area_quad = np.ascontiguousarray(area_quad, dtype=np.float64)
    detj = np.ascontiguousarray(detj, dtype=np.float64)
    Ua = np.ascontiguousarray(Ua, dtype=np.float64)
    Ub = np.ascontiguousarray(Ub, dtype=np.float64)
    K, Np = Ua.shape[0], Ua.shape[1]
    out = np.empty(4)
    lib().vto_l2_state_error(K, Np, area_quad.shape[0], _d(basis_q), _d(area_quad), _d(detj),
                             _d(Ua), _d(Ub), _d(out))
    return out


def totals(basis_q, area_quad, detj, U) -> np.ndarray:
    basis_q = np.ascontiguousarray(basis_q, dtype=np.float64)
    area_quad = np.ascontiguousarray(area_quad, dtype=np.float64)
    detj = np.ascontiguousarray(detj, dtype=np.float64)
    U = np.ascontiguousarray(U, dtype=np.float64)
    out = np.empty(4)
    lib().vto_totals(U.shape[0], U.shape[1], area_quad.shape[0], _d(basis_q), _d(area_quad),
                     _d(detj), _d(U), _d(out))
    return out
