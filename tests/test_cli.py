"""The command line's parser and exit codes (Options.swift:60-154,
Exit.swift:5-18), on the CPU: nothing here touches a GPU."""
import subprocess
import sys

import pytest

from gargantua_b200 import cli


def test_defaults_follow_the_reference():
    o = cli.parse([])
    assert o.command == "interactive" and o.preset == "default" and o.seed == 1
    assert (o.width, o.height) == (3840, 2160) and o.spin == 0.0 and o.strategy == "march"
    assert o.configuration == (1_000_000, 128, 960, 540)


def test_still_with_overrides():
    o = cli.parse(["--still", "x.png", "--width", "640", "--height", "360", "--spin", "0.9", "--camera",
                   "1.0,0.4,40", "--seed", "18446744073709551615", "--preset", "small", "--volume", "192",
                   "--sequence", "3"])
    assert o.command == "still" and o.still_path == "x.png"
    assert (o.width, o.height, o.spin, o.camera, o.sequence) == (640, 360, 0.9, (1.0, 0.4, 40.0), 3)
    assert o.seed == 2**64 - 1
    assert o.configuration == (250_000, 192, 640, 360)


@pytest.mark.parametrize("argv,fragment", [
    (["--preset", "huge"], "unknown preset"),
    (["--volume", "100"], "volume must be"),
    (["--seed", "-1"], "seed must be"),
    (["--seed", str(2**64)], "seed must be"),
    (["--strategy", "trace"], "unknown strategy"),
    (["--fps-cap", "45"], "fps cap"),
    (["--width", "0"], "positive integer"),
    (["--spin", "0.999"], "spin must be"),
    (["--camera", "1,2,60"], "camera needs"),
    (["--camera", "1,2"], "camera needs"),
    (["--still"], "needs a value"),
    (["--frobnicate"], "unknown argument"),
])
def test_refusals(argv, fragment):
    with pytest.raises(cli.UsageError, match=fragment):
        cli.parse(argv)


def test_camera_clamps_elevation():
    cam = cli.orbit_camera(cli.parse(["--camera", "0.5,3.0,30"]))
    assert cam.elevation == 1.5 and cam.distance == 30.0 and cam.azimuth == 0.5


def _run(*args, env=None):
    return subprocess.run([sys.executable, "-m", "gargantua_b200", *args], capture_output=True, text=True,
                          cwd=cli.os.path.dirname(cli.os.path.dirname(cli.__file__)),
                          env=None if env is None else {**cli.os.environ, **env})


def test_exit_codes_and_simple_commands():
    r = _run("--volume", "7")
    assert r.returncode == 64 and "volume must be" in r.stderr
    r = _run("version")
    assert r.returncode == 0 and r.stdout.startswith("gargantua-b200 ")
    r = _run("constants")
    assert r.returncode == 0 and "#define STEP_CAP_STILL" in r.stdout
    r = _run()
    assert r.returncode == 2 and "display" in r.stderr
    r = _run("validate", env={"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode == 2 and "No CUDA device" in r.stderr


def test_request_output_buffers_are_checked_before_the_library_writes():
    import numpy as np
    import pytest

    from gargantua_b200.host import check_pixel_buffer

    check_pixel_buffer(np.zeros((6, 4), np.float16), 6)
    with pytest.raises(ValueError):
        check_pixel_buffer(np.zeros((5, 4), np.float16), 6)
    with pytest.raises(TypeError):
        check_pixel_buffer(np.zeros((6, 4), np.float32), 6)
    with pytest.raises(ValueError):
        check_pixel_buffer(np.zeros((6, 8), np.float16)[:, ::2], 6)
    frozen = np.zeros((6, 4), np.float16)
    frozen.flags.writeable = False
    with pytest.raises(ValueError):
        check_pixel_buffer(frozen, 6)


def test_host_writers_refuse_arrays_of_the_wrong_size():
    import numpy as np
    import pytest

    from gargantua_b200.host import expect_size, write_png

    expect_size(np.zeros((4, 8)), 32, "records")
    with pytest.raises(ValueError, match="31 values given, 32 expected"):
        expect_size(np.zeros(31), 32, "records")
    with pytest.raises(ValueError):
        write_png("unused.png", np.zeros((4, 4), np.uint8))


def test_counters_line_is_the_huds():
    """Renderer.swift:133-137: percent over the drift budget, exhausted and
    captured rays; nothing for a frame with no rays."""
    from gargantua_b200 import types as T

    c = T.MarchCounters(rays=2000, overDriftBudget=31, exhausted=4, captured=250)
    assert cli.counters_line(c) == "drift over budget 1.55 percent, 4 exhausted, 250 captured"
    assert cli.counters_line(T.MarchCounters()) is None
