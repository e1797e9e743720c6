"""Headless CLI (wcsph_headless): the reference's flags and their errors
(parse_cli src/cli.cu:49-101); argument errors need no GPU."""
import subprocess
from pathlib import Path

import pytest

import conftest

CLI = Path(__file__).resolve().parent.parent / "fluid-simulation_b200" / "bin" / "wcsph_headless"


def run(*args):
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=120)


def test_help_lists_the_reference_flags():
    r = run("--help")
    assert r.returncode == 0
    for flag in ("--headless", "--snapshot-load", "--snapshot-save", "--frozen-config", "--searcher",
                 "--tuning-budget", "--stop iters=N | sim-time=T | wall-time=T", "--fixed-dt", "--warmup-iters",
                 "--ktt-output", "--log-csv", "--log-metrics", "--scene"):
        assert flag in r.stderr


@pytest.mark.parametrize("args,msg", [
    (["--bogus"], "Unknown argument: --bogus"),
    (["--headless"], "--stop is required in --headless mode"),
    (["--stop", "iters"], "--stop must be iters=N, sim-time=T, or wall-time=T"),
    (["--stop", "iters=abc"], "Invalid --stop value: abc"),
    (["--stop", "laps=3"], "Unknown --stop kind: laps"),
    (["--searcher", "anneal", "--stop", "iters=1"], "Unknown searcher: anneal"),
    (["--fixed-dt"], "--fixed-dt requires an argument"),
    (["--scene", "dragon_collision", "--headless", "--stop", "iters=1"], "unknown or unavailable scene"),
])
def test_argument_errors(args, msg):
    r = run(*args)
    assert r.returncode == 1
    assert msg in r.stderr


def test_valid_run_without_gpu_fails_cleanly():
    if conftest.HAS_GPU:
        pytest.skip("has a GPU")
    r = run("--scene", "surface_tension", "--headless", "--stop", "iters=2")
    assert r.returncode == 1 and "no CUDA device" in r.stderr.lower() or "cuda" in r.stderr.lower()
