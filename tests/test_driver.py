"""The C++ host driver (kaiju_b200/driver/gamera_gpu_x.cpp) runs the step through the C ABI alone."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "kaiju_b200", "driver", "gamera_gpu_x")


@pytest.fixture(scope="module")
def driver():
    from kaiju_b200 import build as kb
    kb.build()
    return DRIVER


def test_driver_builds_and_rejects_bad_options(driver):
    r = subprocess.run([driver, "--no-such-option"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown option" in r.stderr


@pytest.mark.gpu
def test_driver_blast_wave_matches_oracle(driver, oracle_lib, tmp_path):
    """Warped 16^3 blast wave: three steps through gamera_gpu_x vs the oracle (relative L-inf <= 1e-10)."""
    out = tmp_path / "gas.bin"
    r = subprocess.run([driver, "--problem", "bw", "--n", "16", "--steps", "3", "--ts-out", "1", "--dump", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("ts = ") == 3 and '"zone_updates_per_s_device"' in r.stdout
    gas = np.fromfile(out, dtype=np.float64).reshape((24, 24, 24, 5), order="F")
    o = oracle_lib.Oracle(16, 16, 16, ic="BW", grid="warp", warp_amp=0.04, bounds=(-0.5, 0.5) * 3,
                          CFL=float(np.float32(0.3)), bc=[1] * 6)
    o.step(3)
    ref = o.get("gas")
    for v in range(5):
        den = max(np.abs(ref[..., v]).max(), np.sqrt(np.abs(ref[..., 0]).max() * np.abs(ref[..., 4]).max()))
        assert np.abs(gas[..., v] - ref[..., v]).max() / den <= 1e-10, v
