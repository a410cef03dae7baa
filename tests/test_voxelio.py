"""The reference's binary density format: header of three int32 cell counts, then
float32 cells in lexicographic order (x fastest)."""
import numpy as np
import pytest

from homo3d_b200.voxelio import read_density, write_density


def test_round_trip_and_layout(tmp_path):
    reso = (4, 3, 2)
    rho = np.arange(24, dtype=np.float32) / 24
    p = tmp_path / "rho.bin"
    write_density(p, rho, reso)
    raw = p.read_bytes()
    assert len(raw) == 12 + 4 * 24
    assert np.frombuffer(raw[:12], "<i4").tolist() == [4, 3, 2]
    # cell (x, y, z) = (1, 2, 1) sits at x + 4 (y + 3 z) = 21
    assert np.frombuffer(raw[12:], "<f4")[21] == rho[21]
    back, r = read_density(p)
    assert r == reso and np.array_equal(back, rho)


def test_incomplete_and_bad_files_raise(tmp_path):
    p = tmp_path / "short.bin"
    p.write_bytes(np.asarray([2, 2, 2], "<i4").tobytes() + np.zeros(7, "<f4").tobytes())
    with pytest.raises(ValueError):
        read_density(p)
    q = tmp_path / "bad.bin"
    q.write_bytes(np.asarray([0, 2, 2], "<i4").tobytes())
    with pytest.raises(ValueError):
        read_density(q)
    with pytest.raises(ValueError):
        write_density(tmp_path / "x.bin", np.zeros(5), (2, 2, 2))
