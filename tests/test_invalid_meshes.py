"""Meshes the reference's generator builds but cannot run: with a single row of
cells its periodic vertical-neighbour formula (Meshgeneration.cpp:94-117)
gives every even element a negative neighbour index, which the reference then
reads out of bounds. Every entry point that takes a mesh rejects it on the
host, before any device work (so these run without a GPU)."""
import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def vt():
    return load_package()


@pytest.mark.parametrize("nx", [1, 2, 5])
def test_single_row_mesh_is_rejected(vt, nx):
    pb = vt.Problem(vt.make_params(nx, 1, p=2, integration_order=6))
    conn = pb.array("conn")
    assert (conn < 0).any()  # what the reference's generator produces
    with pytest.raises(vt.VortexError) as ei:
        vt.Solver(pb)
    assert ei.value.status == vt.VT_ERR_INVALID
    with pytest.raises(vt.VortexError) as ej:
        vt.Batch([vt.Problem(vt.make_params(4, 4, p=1, integration_order=4)), pb])
    assert ej.value.status == vt.VT_ERR_INVALID
    with pytest.raises(vt.VortexError) as ek:
        vt.Solver.structured(vt.make_params(nx, 1, p=2, integration_order=6))
    assert ek.value.status == vt.VT_ERR_INVALID


def test_single_column_mesh_is_valid(vt):
    """One column of cells wraps correctly: every neighbour is in range."""
    pb = vt.Problem(vt.make_params(1, 3, p=1, integration_order=4))
    conn = pb.array("conn")
    assert conn.min() >= 0 and conn.max() < pb.K
    # a closed triangulation: every element is across a face from exactly three
    assert (np.bincount(conn.ravel(), minlength=pb.K) == 3).all()
