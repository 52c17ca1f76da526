"""MAT-file reading and writing (no GPU): the reference's data file layout (img, and the structs
atlas / atlas_label whose fields are the atlas volumes) and its result file, against scipy.io's
own level-5 reader and writer, compressed and not."""
import numpy as np
import pytest

import pseudoctimaging_b200 as pct

sio = pytest.importorskip("scipy.io")


def row_based(vol_f):
    """MATLAB [nx ny nz] (column-major) -> the reference's [z][x][y] (ConvertToRowBased)."""
    return np.ascontiguousarray(np.transpose(vol_f, (2, 0, 1)))


def make_data(rng, nx, ny, nz, num):
    img = rng.normal(300, 80, (nx, ny, nz)).astype(np.float32)
    atlas = {f"MRI{i + 1}": rng.normal(300, 80, (nx, ny, nz)).astype(np.float32) for i in range(num)}
    label = {f"MRI{i + 1}": rng.uniform(-1000, 2000, (nx, ny, nz)).astype(np.float32)
             for i in range(num)}
    return img, atlas, label


@pytest.mark.parametrize("compress", [False, True])
@pytest.mark.parametrize("shape,num", [((7, 5, 4), 3), ((16, 9, 6), 1), ((3, 4, 2), 12)])
def test_read_reference_layout(tmp_path, compress, shape, num):
    rng = np.random.default_rng(num)
    img, atlas, label = make_data(rng, *shape, num)
    path = tmp_path / "data.mat"
    sio.savemat(path, {"atlas": atlas, "atlas_label": label, "img": img},
                do_compression=compress, format="5")
    got_img, got_atl, got_ct = pct.read_mat(path)
    assert got_img.shape == (shape[2], shape[0], shape[1])
    assert np.array_equal(got_img, row_based(img))
    for i in range(num):  # atlas i = field i
        assert np.array_equal(got_atl[i], row_based(atlas[f"MRI{i + 1}"]))
        assert np.array_equal(got_ct[i], row_based(label[f"MRI{i + 1}"]))


def test_variable_order_and_other_variables(tmp_path):
    """img may come first; structs with other names are ignored (the reference's Choice)."""
    rng = np.random.default_rng(5)
    img, atlas, label = make_data(rng, 6, 5, 4, 2)
    path = tmp_path / "data.mat"
    sio.savemat(path, {"img": img, "meta": {"a": np.float32(1.0)}, "atlas": atlas,
                       "atlas_label": label}, format="5")
    got_img, got_atl, _ = pct.read_mat(path)
    assert np.array_equal(got_img, row_based(img))
    assert np.array_equal(got_atl[1], row_based(atlas["MRI2"]))


@pytest.mark.parametrize("compress", [False, True])
def test_rejects_malformed(tmp_path, compress):
    rng = np.random.default_rng(1)
    img, atlas, label = make_data(rng, 6, 5, 4, 2)
    bad = dict(label)
    bad["MRI2"] = rng.normal(size=(6, 5, 3)).astype(np.float32)  # wrong size
    path = tmp_path / "bad.mat"
    sio.savemat(path, {"atlas": atlas, "atlas_label": bad, "img": img},
                do_compression=compress, format="5")
    with pytest.raises(pct.PctError):
        pct.read_mat(path)
    no_label = tmp_path / "nolabel.mat"
    sio.savemat(no_label, {"atlas": atlas, "img": img}, format="5")
    with pytest.raises(pct.PctError):
        pct.read_mat(no_label)
    trunc = tmp_path / "trunc.mat"
    trunc.write_bytes(path.read_bytes()[:300])
    with pytest.raises(pct.PctError):
        pct.read_mat(trunc)
    v73 = bytearray(path.read_bytes())  # a version 7.3 header (HDF5 files) is refused
    v73[124:126] = b"\x00\x02"
    (tmp_path / "v73.mat").write_bytes(bytes(v73))
    with pytest.raises(pct.PctError):
        pct.read_mat(tmp_path / "v73.mat")
    with pytest.raises(pct.PctError):
        pct.read_mat(tmp_path / "missing.mat")


def test_write_result_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    vol = rng.normal(size=(5, 7, 6)).astype(np.float32)  # [z][x][y]
    vol[1, 2, 3] = np.nan
    path = tmp_path / "result.mat"
    pct.write_mat(path, "Subject_08_result", vol)
    m = sio.loadmat(path)
    got = m["Subject_08_result"]
    assert got.dtype == np.float32 and got.shape == (7, 6, 5)  # [nx ny nz]
    assert np.array_equal(row_based(got), vol, equal_nan=True)


def test_write_rejects_bad_arguments(tmp_path):
    vol = np.zeros((2, 3, 4), np.float32)
    for name in ("", "x" * 64):
        with pytest.raises(pct.PctError):
            pct.write_mat(tmp_path / "a.mat", name, vol)
    with pytest.raises(pct.PctError):  # unwritable path
        pct.write_mat(tmp_path / "missing_dir" / "a.mat", "v", vol)
