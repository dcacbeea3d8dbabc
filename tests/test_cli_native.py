"""The C++ command-line host (gargantua_b200/cli/gargantua): the reference's
options, refusals and exit codes (Options.swift:60-154, Exit.swift:5-18)
on the CPU; a small still on a GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gargantua_b200", "cli", "gargantua")


@pytest.fixture(scope="module")
def exe():
    subprocess.run(["make", "-s", "-C", os.path.dirname(EXE)], check=True)
    return EXE


def run(exe, *args, env=None):
    return subprocess.run([exe, *args], capture_output=True, text=True,
                          env=None if env is None else {**os.environ, **env})


@pytest.mark.parametrize("argv,fragment", [
    (["--preset", "huge"], "unknown preset"),
    (["--volume", "100"], "volume must be"),
    (["--seed", "-1"], "seed must be"),
    (["--seed", "18446744073709551616"], "seed must be"),
    (["--strategy", "trace"], "unknown strategy"),
    (["--fps-cap", "45"], "fps cap"),
    (["--width", "0"], "positive integer"),
    (["--spin", "0.999"], "spin must be"),
    (["--camera", "1,2,60"], "camera needs"),
    (["--still"], "needs a value"),
    (["--frobnicate"], "unknown argument"),
])
def test_usage_errors_exit_64(exe, argv, fragment):
    r = run(exe, *argv)
    assert r.returncode == 64 and fragment in r.stderr


def test_version_constants_and_operational_exits(exe):
    r = run(exe, "version")
    assert r.returncode == 0 and r.stdout.startswith("gargantua-b200 ")
    r = run(exe, "constants")
    with open(os.path.join(ROOT, "include", "gargantua_constants.h")) as fh:
        assert r.returncode == 0 and r.stdout == fh.read()
    r = run(exe)
    assert r.returncode == 2 and "display" in r.stderr
    r = run(exe, "validate", env={"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode == 2 and "No CUDA device" in r.stderr
    r = run(exe, "--seed", "18446744073709551615", "version")
    assert r.returncode == 0


@pytest.mark.gpu
def test_still_writes_a_png(exe, tmp_path):
    out = tmp_path / "still.png"
    r = run(exe, "--still", str(out), "--width", "320", "--height", "180", "--preset", "small", "--spin", "0.5",
            "--camera", "1.0,0.4,40", "--sequence", "2")
    assert r.returncode == 0, r.stderr
    data = out.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n" and len(data) > 1000
    assert (tmp_path / "seq-000.png").exists() and (tmp_path / "seq-001.png").exists()
    assert "served 320 by 180" in r.stdout
    assert r.stdout.count("drift over budget") == 3  # the still and each of the 2 frames (the HUD's line)


@pytest.mark.gpu
def test_validate_runs_the_goldens_without_the_oracle(exe):
    """`gargantua validate` (Validate.swift:17-55): the eight goldens that need
    no FP64 oracle pass through the C ABI (exit 0); parity, beaming and sky,
    which compare against the oracle, are left to the test suite."""
    r = run(exe, "validate")
    assert r.returncode == 0, r.stdout + r.stderr
    rows = {line.split()[0]: line.split()[-1] for line in r.stdout.splitlines()[2:] if line.strip()}
    run_by_host = ["isco", "determinism", "shadow", "deflection", "conservation_interactive", "conservation_still",
                   "jump", "shadow_kerr"]
    assert all(rows[name] == "pass" for name in run_by_host), rows
    assert all(rows[name] == "skipped" for name in ("parity", "beaming", "sky")), rows
