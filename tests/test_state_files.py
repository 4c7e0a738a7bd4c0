"""Full-precision state files (vt_write_state_file / vt_read_state_file, the
format of vt_save_state): round trip and rejection of damaged files, no GPU."""
import numpy as np
import pytest


def test_round_trip_is_exact(vt, tmp_path):
    rng = np.random.default_rng(0)
    U = rng.standard_normal((37, 10, 4)) * 1e3
    path = str(tmp_path / "s.vts")
    vt.write_state_file(path, 3, U, time=1.2345678901234567)
    V, p, t = vt.read_state_file(path)
    assert p == 3 and t == 1.2345678901234567
    np.testing.assert_array_equal(V, U)
    raw = open(path, "rb").read()
    assert raw[:8] == b"VTSTATE\0" and len(raw) == 32 + U.nbytes


@pytest.mark.parametrize("damage", ["magic", "truncated", "longer", "np"])
def test_damaged_files_are_rejected(vt, tmp_path, damage):
    U = np.ones((5, 6, 4))
    path = str(tmp_path / "s.vts")
    vt.write_state_file(path, 2, U)
    raw = bytearray(open(path, "rb").read())
    if damage == "magic":
        raw[0] = ord("X")
    elif damage == "truncated":
        raw = raw[:-8]
    elif damage == "longer":
        raw += b"\0" * 8
    else:
        raw[20:24] = (7).to_bytes(4, "little")  # Np field no longer matches p
    open(path, "wb").write(bytes(raw))
    with pytest.raises(vt.VortexError):
        vt.read_state_file(path)
