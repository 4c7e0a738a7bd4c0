"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources are mounted (the fixtures are committed, so the
tests themselves never need the sources):

    make -C oracle ref            # builds oracle/_ref/vt_ref_harness
    python tests/golden/make_golden.py

Every case runs the reference's own code (compiled from its sources by
oracle/Makefile; only main.cpp and the text-output Utilities.cpp are replaced by
oracle/ref_harness.cpp) and stores its full-precision dumps as one compressed
.npz per case. The reference has no tests of its own, so these fixtures are the
known answers that pin the oracle and the product's host precompute.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "vt_ref_harness")
SHIPPED_INPUT = os.path.join(os.environ.get("VT_REFERENCE_SRC", "/root/reference"), "input_files", "input")

# name -> harness arguments
CASES = {
    # config 1 mesh (8x8 cells, p=3, io=10), one RK4 step, RHS of the IC
    "c1_p3_io10_rk4_1step": ["--steps", "1", "--rhs"],
    # the shipped input file itself (io=6), one RK4 step
    "shipped_p3_io6_rk4_1step": ["--input", SHIPPED_INPUT, "--steps", "1", "--rhs", "--no-ops"],
    # perturbed (float perturb_grid) and non-square meshes, all orders, both steppers
    "p3_io10_16x16_pert_rk4": ["--nx", "16", "--ny", "16", "--perturb", "0.2", "--dt", "1e-3",
                               "--steps", "3", "--rhs", "--no-ops", "--dump-every", "1"],
    "p2_io6_12x8_pert_fe": ["--nx", "12", "--ny", "8", "--p", "2", "--io", "6", "--perturb", "0.2",
                            "--stepping", "0", "--dt", "5e-4", "--steps", "5", "--rhs", "--no-ops"],
    "p1_io10_16x16_pert_rk4": ["--nx", "16", "--ny", "16", "--p", "1", "--perturb", "0.2",
                               "--dt", "2e-3", "--steps", "4", "--rhs", "--no-ops"],
    "p0_io2_8x8_rk4": ["--p", "0", "--io", "2", "--dt", "1e-3", "--steps", "3", "--rhs", "--no-ops"],
    "p2_io10_8x8_l2proj_rk4": ["--p", "2", "--init-type", "1", "--dt", "1e-3", "--steps", "2",
                               "--rhs", "--no-ops"],
    "p3_io8_10x6_pert_rk4": ["--nx", "10", "--ny", "6", "--io", "8", "--perturb", "0.15",
                             "--domain-x", "7.5", "--domain-y", "4.5", "--dt", "4e-4",
                             "--steps", "2", "--rhs", "--no-ops"],
    # config 1 in full: 10000 RK4 steps over T = 10*sqrt(2), states every 2500 steps
    "c1_p3_io10_rk4_10000": ["--steps", "10000", "--no-ops", "--dump-every", "2500"],
}

INT_FILES = ("conn", "type")


def run_case(name: str, args: list[str]) -> str:
    tmp = tempfile.mkdtemp(prefix="vt_golden_")
    cmd = [HARNESS, *args, "--dump", tmp]
    env = dict(os.environ, OMP_SCHEDULE="static")
    subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    arrays = {}
    meta = json.load(open(os.path.join(tmp, "meta.json")))
    for fn in sorted(os.listdir(tmp)):
        base, ext = os.path.splitext(fn)
        if ext == ".f64":
            arrays[base] = np.fromfile(os.path.join(tmp, fn), dtype="<f8")
        elif ext == ".i32":
            arrays[base] = np.fromfile(os.path.join(tmp, fn), dtype="<i4")
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    arrays["args"] = np.frombuffer(json.dumps(args).encode(), dtype=np.uint8)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, **arrays)
    shutil.rmtree(tmp)
    return out


def quadrature_tables() -> str:
    """Line and area rules the reference selects for integration_order 0..19
    (Quadraturerule.cpp:125-126, :590-591), plus M^-1_ref and S_ref for p=0..3."""
    arrays = {}
    for io in range(20):
        for p in range(4):
            tmp = tempfile.mkdtemp(prefix="vt_quad_")
            subprocess.run([HARNESS, "--nx", "2", "--ny", "2", "--p", str(p), "--io", str(io),
                            "--steps", "0", "--no-ops", "--dump", tmp], check=True,
                           stdout=subprocess.DEVNULL)
            if p == 0:
                arrays[f"line_{io}"] = np.fromfile(os.path.join(tmp, "line_quad.f64"))
                arrays[f"area_{io}"] = np.fromfile(os.path.join(tmp, "area_quad.f64"))
            arrays[f"minv_{io}_{p}"] = np.fromfile(os.path.join(tmp, "minv_ref.f64"))
            arrays[f"stiff_{io}_{p}"] = np.fromfile(os.path.join(tmp, "stiff_ref.f64"))
            arrays[f"phi_plus_{io}_{p}"] = np.fromfile(os.path.join(tmp, "phi_plus.f64"))
            arrays[f"phi_minus_{io}_{p}"] = np.fromfile(os.path.join(tmp, "phi_minus.f64"))
            arrays[f"nodes_ref_{p}"] = np.fromfile(os.path.join(tmp, "nodes_ref.f64"))
            shutil.rmtree(tmp)
    out = os.path.join(HERE, "quadrature_tables.npz")
    np.savez_compressed(out, **arrays)
    return out


def main() -> int:
    if not os.path.exists(HARNESS):
        print("build the harness first: make -C oracle ref", file=sys.stderr)
        return 1
    only = set(sys.argv[1:])
    if not only or "quadrature_tables" in only:
        out = quadrature_tables()
        print(f"quadrature_tables: {os.path.getsize(out) / 1024:.1f} KiB")
    for name, args in CASES.items():
        if only and name not in only:
            continue
        out = run_case(name, args)
        print(f"{name}: {os.path.getsize(out) / 1024:.1f} KiB")
    return 0


if __name__ == "__main__":
    sys.exit(main())
