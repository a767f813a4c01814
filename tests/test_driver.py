"""The command-line driver (reference CLI and time loop over the C ABI)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "turbchannel_b200", "turbch_run")


@pytest.fixture(scope="module")
def exe():
    from turbchannel_b200 import build

    build.build()
    return EXE


def test_driver_help_lists_reference_options(exe):
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    for opt in ["--device", "--nz", "--TimeMax", "--TimeStartAveraging", "--TimeStepsMax", "--tau", "--CFLmin",
                "--CFLmax", "--SProgress", "--FProgress", "--PProgress"]:
        assert opt in r.stdout


def test_driver_rejects_unknown_option(exe):
    r = subprocess.run([exe, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["hw2", "vv4", "colloc"])
def test_driver_runs_constant_flow_rate(exe, tmp_path, scheme):
    nz = "25" if scheme == "colloc" else "24"
    r = subprocess.run([exe, "--scheme", scheme, "--nx", "32", "--ny", "16", "--nz", nz, "--TimeStepsMax", "30",
                        "--tau", "0.002", "--CFLmin", "0", "--CFLmax", "1e30", "--cfr", "-s", "10", "-a", "0",
                        "-p", "20"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    rows = [list(map(float, l.split())) for l in open(tmp_path / "log.dat")]
    assert len(rows) == 4
    assert all(abs(row[1] - 1.0) < 1e-9 for row in rows)  # bulk velocity held by the flow-rate forcing
    assert (tmp_path / "res.dat").exists() and (tmp_path / "r00020.dat").exists()
