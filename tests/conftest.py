"""Shared test helpers: golden fixtures, the oracle binding, the product package."""
from __future__ import annotations

import glob
import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    """Import vortex-transport_b200/ (a directory name that is not an identifier)."""
    name = "vortex_transport_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "vortex-transport_b200")
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class Golden:
    """One fixture written by tests/golden/make_golden.py from the reference."""

    def __init__(self, path: str):
        self.path = path
        self.name = os.path.splitext(os.path.basename(path))[0]
        self._z = np.load(path)
        self.meta = json.loads(bytes(self._z["meta"]).decode())
        self.args = json.loads(bytes(self._z["args"]).decode())
        self.K, self.Np, self.p = self.meta["K"], self.meta["Np"], self.meta["p"]
        self.nfq = self.meta["nfq"]

    def __contains__(self, key):
        return key in self._z

    def __getitem__(self, key):
        a = self._z[key]
        K, Np, nfq = self.K, self.Np, self.nfq
        shapes = {
            "vertices": (K, 3, 2), "conn": (K, 3), "type": (K,), "nodes_ref": (Np, 2),
            "line_quad": (nfq, 2), "area_quad": (-1, 3), "minv_ref": (Np, Np),
            "stiff_ref": (2, Np, Np), "jac": (K, 4), "jinv": (K, 4), "detj": (K,),
            "detjinv": (K,), "normals": (K, 3, 2), "sides": (K, 3), "nodes_phys": (K, Np, 2),
            "minv_phys": (K, Np, Np), "stiff_phys": (K, 2, Np, Np),
            "phi_plus": (3, Np, nfq), "phi_minus": (3, Np, nfq),
            "F0": (K, Np, 2, 4), "F_final": (K, Np, 2, 4),
        }
        if key in shapes:
            return a.reshape(shapes[key])
        if key.startswith("U") or key == "rhs0":
            return a.reshape(K, Np, 4)
        return a

    def oracle_mesh(self):
        import vt_oracle
        return vt_oracle.OracleMesh(self.p, self["vertices"], self["conn"], self["type"],
                                    self["minv_ref"], self["stiff_ref"], self["phi_plus"],
                                    self["phi_minus"], self["line_quad"])


def golden_paths():
    """Problem fixtures (the quadrature table fixture has its own test)."""
    return sorted(p for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz"))
                  if not p.endswith("quadrature_tables.npz"))


def golden(name: str) -> Golden:
    return Golden(os.path.join(GOLDEN_DIR, name + ".npz"))


@pytest.fixture(scope="session")
def vt():
    return load_package()
