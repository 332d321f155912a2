"""The standalone C++ driver (driver/monalisa_driver.cpp) without a GPU: it
is built, prints its usage, and resolves a JSON configuration with
command-line overrides (--dry-run touches no device)."""
import json
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "driver", "_bin", "monalisa_driver")


def _driver():
    from monalisa_b200 import build

    build.build()
    assert os.access(DRIVER, os.X_OK), DRIVER
    return DRIVER


def test_driver_usage():
    r = subprocess.run([_driver(), "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "usage: monalisa_driver" in r.stdout


def test_driver_config_and_overrides(tmp_path):
    cfg = tmp_path / "cfg.json"
    cfg.write_text(json.dumps({"synthetic": "koosh3d", "n": 32, "kernelParam": [0.61, 10], "nCGD": 10,
                               "kernel": "gauss"}))
    r = subprocess.run([_driver(), "--config", str(cfg), "--nCGD", "5", "--dry-run"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    got = dict(line.split(" = ", 1) for line in r.stdout.strip().splitlines())
    assert got["synthetic"] == "koosh3d" and got["n"] == "32" and got["nCGD"] == "5"
    assert got["kernelParam"] == "0.61,10"


def test_driver_rejects_bad_arguments():
    r = subprocess.run([_driver(), "--traj"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "bad argument" in r.stderr
