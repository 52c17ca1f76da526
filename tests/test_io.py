"""Volume file formats of the drop-in command line (host side, no GPU)."""
import numpy as np
import pytest

import pseudoctimaging_b200 as pct


def test_matrixio_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(0)
    vol = (rng.standard_normal((2, 5, 4, 3)) * 1e3).astype(np.float32)
    p = tmp_path / "v.txt"
    pct.write_matrixio(p, vol)
    back = pct.read_matrixio(p)
    assert back.shape == (2, 5, 4, 3)
    assert np.array_equal(back.view(np.uint32), vol.view(np.uint32))


def test_matrixio_reads_the_reference_writer_output(tmp_path):
    """MatrixIO<T>::Store writes num, rows, cols, depth on four lines, then all values on one
    line separated by spaces with 6 significant digits (PatchBasedPseudoCT.cu:781-805)."""
    vals = np.arange(2 * 3 * 4, dtype=np.float32) * np.float32(0.125) - 1
    p = tmp_path / "ref.txt"
    p.write_text("1\n3\n4\n2\n" + " ".join(f"{v:g}" for v in vals) + " ")
    back = pct.read_matrixio(p)
    # rows=3 (nx), cols=4 (ny), depth=2 (nz): [num][depth][rows][cols]
    assert back.shape == (1, 2, 3, 4)
    np.testing.assert_array_equal(back.reshape(-1), vals)


def test_matrixio_rejects_short_or_bad_files(tmp_path):
    p = tmp_path / "short.txt"
    p.write_text("1\n2\n2\n2\n1 2 3\n")
    with pytest.raises(pct.PctError):
        pct.read_matrixio(p)
    q = tmp_path / "hdr.txt"
    q.write_text("1\nx\n2\n2\n")
    with pytest.raises(pct.PctError):
        pct.read_matrixio(q)
    with pytest.raises(pct.PctError):
        pct.read_matrixio(tmp_path / "missing.txt")


def test_raw_round_trip_and_size_check(tmp_path):
    v = np.linspace(-5, 5, 60, dtype=np.float32)
    p = tmp_path / "v.f32"
    assert pct.lib.pct_raw_write(str(p).encode(), v.ctypes.data, v.size) == 0
    out = np.empty_like(v)
    assert pct.lib.pct_raw_read(str(p).encode(), out.ctypes.data, out.size) == 0
    assert np.array_equal(out, v)
    small = np.empty(10, np.float32)
    assert pct.lib.pct_raw_read(str(p).encode(), small.ctypes.data, small.size) == -1
