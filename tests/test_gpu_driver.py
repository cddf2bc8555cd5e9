"""The command-line driver (the X/main.cpp replacement) end to end: parameter file,
pair-index list, TIFF frames in, the five Tecplot files per pair out, with the
reference's messages and exit status; and the same fields as the C-ABI engine."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "piv_xcorr2d_v1.0_b200" / "lib" / "piv_xcorr2d"


def write_setup(tmp, pairs, Nx=320, Ny=256):
    (tmp / "img").mkdir()
    for k, idx in enumerate(pairs):
        s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_UNIFORM, a=2.2 + 0.3 * k, b=-1.1, seed=100 + k)
        f1, f2 = P.synth_pair(s)
        for name, img in ((f"1_{idx:04d}.tif", f1), (f"2_{idx:04d}.tif", f2)):
            assert P.lib().piv_tiff_write8(str(tmp / "img" / name).encode(), img.ctypes.data_as(P._U8), Nx, Ny) == 0
    (tmp / "pairs.txt").write_text("\n".join(str(i) for i in pairs) + "\n")
    lines = [str(tmp / "img" / "1_"), ".tif", str(tmp / "img" / "2_"), ".tif", str(tmp / "pairs.txt"),
             str(tmp / "out") + "/",
             "0", "1", "40", "0.91", str(Nx), str(Ny), "64", "64", "32", "32", "2", "32", "32", "16", "16", "2", "1",
             "5", "5", "2", "5", "2", "2", "3", "3", "1", "5", "5", "2", "5", "2", "2", "3", "3", "1",
             "0.25", "0.25", "0.25", "0.25", "4", "-100", "100", "-100", "100"]
    (tmp / "Parameter.dat").write_text("\r\n".join(lines))
    return tmp / "Parameter.dat"


@pytest.mark.parametrize("overlap", [False, True])
def test_driver_end_to_end(cuda, tmp_path, overlap):
    pairs = [1, 7, 12]
    par = write_setup(tmp_path, pairs)
    cmd = [str(EXE), str(par)] + (["--overlap"] if overlap else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "NO ERROR!" in r.stdout and r.stdout.count("Done!") == len(pairs)
    p, paths = P.read_params(par)
    for idx in pairs:
        for kind in range(5):
            assert Path(P.output_name(p, paths["folder_result"], idx, kind)).exists()
    # the last pair through the C-ABI gives the same grid-2 filtered file
    f1 = np.empty((p.Ny, p.Nx), np.uint8)
    f2 = np.empty_like(f1)
    for name, a in ((f"1_{pairs[-1]:04d}.tif", f1), (f"2_{pairs[-1]:04d}.tif", f2)):
        assert P.lib().piv_tiff_read8(str(tmp_path / "img" / name).encode(), a.ctypes.data_as(P._U8), p.Nx, p.Ny) == 0
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.run_pair()
        mine = tmp_path / "mine.dat"
        e.write_tecplot(mine, 3)
    ref = Path(P.output_name(p, paths["folder_result"], pairs[-1], 3))
    assert mine.read_bytes() == ref.read_bytes()
    lines = ref.read_text().splitlines()
    assert lines[0] == 'TITLE = "B00001"' and lines[2] == 'ZONE T="Frame 0", I=20, J=16'
    dx = np.array([float(l.split("\t")[2]) for l in lines[3:]])
    assert abs(np.median(dx) - 2.8) < 0.1


def test_driver_shards_resume_and_npy(cuda, tmp_path):
    pairs = [2, 3, 5, 8, 13]
    par = write_setup(tmp_path, pairs)
    p, paths = P.read_params(par)
    # two replicas (one GPU here, run one after the other): each takes every other pair
    for r in range(2):
        out = subprocess.run([str(EXE), str(par), "--shard", f"{r}/2", "--npy"], capture_output=True, text=True,
                             timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.count("Done!") == len(pairs[r::2])
    for idx in pairs:
        for kind in range(5):
            dat = Path(P.output_name(p, paths["folder_result"], idx, kind))
            assert dat.exists()
            arr = np.load(dat.with_suffix(".npy"))
            lines = dat.read_text().splitlines()[3:]
            if kind in (0, 2):
                assert arr.shape[2:] == (p.Npeak_save, 2)
                first = np.array([[float(v) for v in l.split("\t")[2:4]] for l in lines])
                assert np.allclose(arr[:, :, 0, :].reshape(-1, 2), first, atol=0.0051)
            else:
                assert arr.shape[2] == 2
                vals = np.array([[float(v) for v in l.split("\t")[2:4]] for l in lines])
                assert np.allclose(arr.reshape(-1, 2), vals, atol=0.0051)
    # everything is there: --resume does nothing
    out = subprocess.run([str(EXE), str(par), "--resume"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and "Resuming: 5 of 5" in out.stdout and "Done!" not in out.stdout
    # one output removed: only that pair runs again
    Path(P.output_name(p, paths["folder_result"], 8, 4)).unlink()
    out = subprocess.run([str(EXE), str(par), "--resume"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and "Resuming: 4 of 5" in out.stdout and out.stdout.count("Done!") == 1
    assert Path(P.output_name(p, paths["folder_result"], 8, 4)).exists()


def test_driver_error_paths(cuda, tmp_path):
    r = subprocess.run([str(EXE), str(tmp_path / "nope.dat")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Can't open parameter file!" in r.stdout
    par = write_setup(tmp_path, [3])
    lines = par.read_bytes().decode().split("\r\n")
    assert len(lines) == 50
    (tmp_path / "short.dat").write_text("\n".join(lines[:41]))
    r = subprocess.run([str(EXE), str(tmp_path / "short.dat")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Parameter missing" in r.stdout
    (tmp_path / "pairs.txt").write_text("3\n4\n")  # pair 4 has no frames
    r = subprocess.run([str(EXE), str(par)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "missing" in r.stdout and "ERROR!" in r.stdout
