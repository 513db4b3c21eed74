"""Run a C++ caller written against the reference's glst_force<double>
interface, linked to this project, and compare with the Python path."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from test_cpp_shim import build_client

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_cpp_client_runs(tmp_path, pkg):
    if not (shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc")):
        pytest.skip("nvcc not available")
    exe = build_client(str(tmp_path))
    stdout = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    # the set-up summary the reference prints from init comes first
    assert "Total number of cubature nodes:" in stdout
    e_sum, e_dev, fx0 = (float(v) for v in stdout.split()[-3:])
    x = [1, 2, 3, 11, 12, 13]
    y = [1, 2, 1, 12, 11, 12]
    z = [1, 1, 2, 13, 12, 11]
    q = [-0.8, 0.4, 0.4, -0.8, 0.4, 0.4]
    with pkg.GlstForce(6, 1e-4, 20.0, 20.0, 20.0, rcut=10.0) as f:
        f.calc_ener_force(*[torch.tensor(v, dtype=torch.float64, device="cuda:0") for v in (x, y, z, q)])
        fx, fy, fz, en = f.get_ef()
    assert e_sum == pytest.approx(0.5 * np.sum(en), rel=1e-14)
    assert e_dev == pytest.approx(e_sum, rel=1e-12)
    assert fx0 == pytest.approx(fx[0], rel=1e-14)


def test_reference_driver_against_this_engine(tmp_path, pkg):
    """The reference's own driver (test/full_example.cu, compiled unchanged
    against include/ by `make -C oracle drivers`), on a water box written as
    CHARMM files; it must run and report an error report."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "oracle", "_ref", "full_example_b200")
    if not os.path.exists(exe):
        pytest.skip("reference driver not built here (needs the reference sources)")
    from glst_b200 import systems
    x, y, z, q = systems.water_box(1000, 31.04, seed=8)
    systems.write_charmm(str(tmp_path / "w"), x, y, z, q)
    r = subprocess.run([exe, "w", "1e-5", "31.04", "8.0"], cwd=str(tmp_path), capture_output=True, text=True,
                       env=dict(os.environ, GLST_BENCH_TERMINAL="1"), timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Total GLST Runtime" in r.stdout and "Root Mean Squared" in r.stdout
