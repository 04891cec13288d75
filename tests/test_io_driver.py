"""Reference file formats and the C++ host driver smectic_run."""
import os
import subprocess

import numpy as np
import pytest

from smectic3d_b200 import io as sio

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "smectic3d_b200", "smectic_run")


def test_psi_text_roundtrip_exact(tmp_path):
    psi = np.random.default_rng(0).standard_normal((8, 8, 8))
    p = tmp_path / "psi.dat"
    sio.write_psi_text(p, psi)
    assert np.array_equal(sio.read_psi_text(p, 8), psi)
    text = p.read_text()
    assert text.count("\n ") == 512  # every value followed by "\n " (periodicFFT/pf3d.cpp:539)


def test_psi_text_reference_precision(tmp_path):
    psi = np.full((4, 4, 4), 1.2441123456)
    p = tmp_path / "psi.dat"
    sio.write_psi_text(p, psi, digits=6)
    assert p.read_text().startswith("1.24411\n ")
    assert np.allclose(sio.read_psi_text(p, 4), 1.24411)


def test_short_psi_file_is_rejected(tmp_path):
    p = tmp_path / "psi.dat"
    p.write_text("1\n 2\n ")
    with pytest.raises(ValueError):
        sio.read_psi_text(p, 2)


def test_surface_files(tmp_path):
    z = np.array([[3, -1], [5, 7]])
    v = np.array([[0.1, np.nan], [0.2, 0.3]])
    n = sio.write_surface_files(tmp_path, z, v, v, v)
    assert n == 3
    assert (tmp_path / "surfPsi.dat").read_text() == "3\n 5\n 7\n "


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")
def test_driver_help_and_bad_option():
    r = subprocess.run([DRIVER, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage" in r.stdout
    for flag in ("--sub-sigma", "--surface-every", "--amp-nw"):
        assert flag in r.stdout
    r = subprocess.run([DRIVER, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2


@pytest.mark.gpu
def test_driver_matches_python_api(tmp_path):
    import smectic3d_b200 as S
    n, steps = 32, 20
    r = subprocess.run([DRIVER, "--n", str(n), "--nw", "8", "--dt", "0.05", "--eps", "-0.7", "--ic", "lamellae",
                        "--l1-every", "10", "--max-steps", str(steps), "--out", str(tmp_path)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    psi0 = sio.read_psi_text(tmp_path / "psiIC.dat", n)
    assert np.allclose(psi0, S.ic.pf3d_lamellae(n, 2 * np.pi / 8), atol=1e-5)
    l1 = sio.read_l1(tmp_path / "L1.dat")
    assert l1.shape == (2,)
    with S.Solver(S.Params(n=n, dt=0.05, eps=-0.7, l1_interval=10)) as s:
        s.set_psi(psi0)
        s.step(steps)
        ref = s.get_psi()
        l1_ref, _ = s.l1()
    got = sio.read_psi_text(tmp_path / "psi.dat", n)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-5)
    assert abs(l1[-1] - l1_ref[0]) <= 1e-5 * abs(l1_ref[0])


@pytest.mark.gpu
def test_driver_neumann_surface_and_amplitude(tmp_path):
    """cosNoAdvMorphCurv-style run: the surface files hold every column at each
    save, psiAvg.dat is the local-amplitude map of the final psi."""
    import smectic3d_b200 as S
    n = 32
    r = subprocess.run([DRIVER, "--n", str(n), "--nw", "8", "--dt", "0.05", "--eps", "-0.7", "--ic", "hyperboloid",
                        "--boundary", "neumann", "--sub-sigma", "0.3", "--sub-z0", "1.5", "--l1-every", "5",
                        "--surface-every", "2", "--max-steps", "20", "--amp-nw", "8", "--alternate",
                        "--save-every", "1", "--out", str(tmp_path)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    z = np.loadtxt(tmp_path / "surfPsi.dat")
    assert z.size == 2 * n * n  # two saves (blocks 2 and 4), every column
    assert np.isfinite(np.loadtxt(tmp_path / "curvH.dat")).all()
    mid = np.loadtxt(tmp_path / "psiMid.dat")
    assert mid.size == 4 * n * n  # one y = N/2 slice per save, four saves
    assert (tmp_path / "psiB.dat").exists()
    psi = sio.read_psi_text(tmp_path / "psi.dat", n)
    assert np.allclose(mid[-n * n:].reshape(n, n), psi[:, n // 2, :], atol=1e-5)  # last save = final state
    amp = sio.read_psi_text(tmp_path / "psiAvg.dat", n)
    from oracle import sh_oracle as O
    ref = O.local_amplitude(psi, 2 * np.pi / 8, 8)
    assert np.allclose(amp, ref, rtol=1e-4, atol=1e-5)  # psi.dat and psiAvg.dat carry 6 digits
