"""The drop-in command line end to end on the GPU: reference argv, config file, MatrixIO volumes
in, regularised HU volume out, compared with the oracle pipeline."""
import subprocess

import numpy as np
import pytest

import oracle
import pseudoctimaging_b200 as pct
from conftest import REPO, load_golden

pytestmark = pytest.mark.gpu
CLI = REPO / "pseudoctimaging_b200" / "bin" / "PatchBasedPseudoCT_b200"


def run_cli(*args):
    res = subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    return res.stdout


def test_cli_matrixio_config_matches_reference_pipeline(tmp_path):
    g = load_golden("nh9_3atlas")
    pct.write_matrixio(tmp_path / "atlas.txt", g["atlas_mri"])
    pct.write_matrixio(tmp_path / "label.txt", g["atlas_ct_hu"])
    pct.write_matrixio(tmp_path / "im.txt", g["img"])
    cfg = tmp_path / "data.cfg"
    cfg.write_text(f"0\n{tmp_path/'atlas.txt'}\n{tmp_path/'label.txt'}\n{tmp_path/'im.txt'}\n")
    out = tmp_path / "result"
    run_cli(cfg, out, 2, 9, 2.5, 1.0, 0)
    got = pct.read_matrixio(str(out) + ".txt")[0]
    ref = g["hu"]
    d = np.abs(got - ref)
    assert d.max() <= 17.0 and (d > 0).mean() < 0.01


def test_cli_synthetic_and_raw_modes(tmp_path):
    cfg = tmp_path / "synth.cfg"
    cfg.write_text("3\n1\n30\n28\n26\n6\n5\n")
    run_cli(cfg, tmp_path / "synth", 3, 7, 2.5, 1.0)
    got = np.fromfile(str(tmp_path / "synth") + ".f32", np.float32).reshape(26, 30, 28)
    s = pct.synth_subject(30, 28, 26, 1, n_blobs=6, seed=5)
    label = pct.normalize_labels(s.atlas_ct)
    fused = oracle.fuse_port(s.img, s.atlas_mri, label, 7, 337.5)
    reg, _ = oracle.regularize_port(fused, 7)
    ref = oracle.finalize_port(reg)
    d = np.abs(got - ref)
    assert d.max() <= 17.0 and (d > 0).mean() < 0.01
    # mode 2: the same volumes as raw files give the same output
    s.atlas_mri.tofile(tmp_path / "a.f32")
    s.atlas_ct.tofile(tmp_path / "c.f32")
    s.img.tofile(tmp_path / "i.f32")
    cfg2 = tmp_path / "raw.cfg"
    cfg2.write_text(f"2\n1\n30\n28\n26\n{tmp_path/'a.f32'}\n{tmp_path/'c.f32'}\n{tmp_path/'i.f32'}\n")
    run_cli(cfg2, tmp_path / "raw", 0, 7, 2.5, 1.0)
    got2 = np.fromfile(str(tmp_path / "raw") + ".f32", np.float32).reshape(26, 30, 28)
    assert np.array_equal(got2, got)


def test_cli_timing_mode_and_usage(tmp_path):
    cfg = tmp_path / "rand.cfg"
    cfg.write_text("1\n2\n24\n24\n20\n")
    out = run_cli(cfg, tmp_path / "t", 4, 7)
    assert out.count("Elapsed Time") == 10
    res = subprocess.run([str(CLI)], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0 and "Usage" in res.stdout


def test_cli_tensor_core_and_learned_choices(tmp_path):
    """EXEC_CHOICE 5, 6 and 7 through the drop-in command line (NH = 11), against choice 3 on the
    same synthetic subject; 7 uses the checkpoint shipped beside the program by default."""
    cfg = tmp_path / "synth.cfg"
    cfg.write_text("3\n2\n34\n37\n30\n8\n17\n")
    outs = {}
    for choice in (3, 5, 6, 7):
        run_cli(cfg, tmp_path / f"c{choice}", choice, 11, 2.5, 1.0)
        outs[choice] = np.fromfile(str(tmp_path / f"c{choice}") + ".f32", np.float32)
    for choice in (5, 6, 7):
        d = np.abs(outs[choice] - outs[3])
        assert np.isfinite(outs[choice]).all()
        assert d.mean() < 5.0, (choice, d.mean())
    res = subprocess.run([str(CLI), str(cfg), str(tmp_path / "bad"), "7", "11"],
                         capture_output=True, text=True, timeout=300,
                         env={"PCT_LEARNED_MODEL": str(tmp_path / "missing.pctl")})
    assert res.returncode != 0 and "missing.pctl" in res.stderr


def test_cli_mat_data_file(tmp_path):
    """The reference's own data-file format: a MAT-file with img and the structs atlas and
    atlas_label (one field per atlas), written here by scipy.io in MATLAB's column-major
    [nx ny nz] layout, compressed; the result comes back as <output>.mat with one single variable
    named after the result. Same output as the raw-file mode on the same volumes."""
    sio = pytest.importorskip("scipy.io")
    s = pct.synth_subject(30, 28, 26, 2, n_blobs=6, seed=9)
    col = lambda v: np.ascontiguousarray(np.transpose(v, (1, 2, 0)))  # [z][x][y] -> [nx ny nz]
    sio.savemat(tmp_path / "Subject.mat", {
        "atlas": {f"MRI{i + 1}": col(s.atlas_mri[i]) for i in range(2)},
        "atlas_label": {f"MRI{i + 1}": col(s.atlas_ct[i]) for i in range(2)},
        "img": col(s.img)}, do_compression=True, format="5")
    run_cli(tmp_path / "Subject.mat", tmp_path / "Subject_result", 2, 7, 2.5, 1.0)
    m = sio.loadmat(tmp_path / "Subject_result.mat")
    got = np.ascontiguousarray(np.transpose(m["Subject_result"], (2, 0, 1)))
    s.atlas_mri.tofile(tmp_path / "a.f32")
    s.atlas_ct.tofile(tmp_path / "c.f32")
    s.img.tofile(tmp_path / "i.f32")
    cfg = tmp_path / "raw.cfg"
    cfg.write_text(f"2\n2\n30\n28\n26\n{tmp_path/'a.f32'}\n{tmp_path/'c.f32'}\n{tmp_path/'i.f32'}\n")
    run_cli(cfg, tmp_path / "raw", 2, 7, 2.5, 1.0)
    ref = np.fromfile(str(tmp_path / "raw") + ".f32", np.float32).reshape(26, 30, 28)
    assert np.array_equal(got, ref)
