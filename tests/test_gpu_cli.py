"""The dtfe program (the reference's example driver, src/main.c:35-195) end
to end on the GPU: its map file and image, reproducible under a fixed seed,
and the map's projected mass against the particle count."""
import numpy as np
import pytest

from test_host_abi import run_cli

pytestmark = pytest.mark.gpu


def test_cli_writes_map_and_image(tmp_path):
    n, G = 3000, 32
    r = run_cli(tmp_path, n=n, G=G)
    assert r.returncode == 0, r.stdout + r.stderr
    rho = np.fromfile(tmp_path / "pts.bin.rho.bin", np.float64)
    assert rho.size == G * G and (rho >= 0).all()
    # a blob well inside the field: the map's integral estimates the mass
    assert abs(rho.sum() / G / G / n - 1.0) < 0.03
    tiff = (tmp_path / "pts.bin.rho.tiff").read_bytes()
    assert tiff[:4] == b"II*\x00" and len(tiff) == 8 + 2 + 12 * 12 + 4 + 1536 + G * G
    again = tmp_path / "again"
    again.mkdir()
    r2 = run_cli(again, n=n, G=G)
    assert r2.returncode == 0
    assert np.array_equal(np.fromfile(again / "pts.bin.rho.bin", np.float64), rho)
