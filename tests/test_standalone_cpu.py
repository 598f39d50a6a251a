"""The native tdmd_standalone's command line without a GPU: version, usage,
the no-data banner and the --morse parse error of the reference driver
(src/drivers/tdmd_main.cpp:46-170); a missing data file is an error exit."""
from __future__ import annotations

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def drivers():
    from tdmd_claude_b200 import build
    try:
        return build.build_driver()
    except (OSError, RuntimeError) as e:  # no host compiler or CUDA headers here
        pytest.skip(f"native driver not buildable: {e}")


@pytest.mark.parametrize("name", ["tdmd_standalone", "tdmd_standalone_mixed"])
def test_native_driver_command_line(drivers, name):
    exe = drivers[name]

    def run(*args):
        return subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)

    r = run("--version")
    assert r.returncode == 0 and r.stdout.startswith("tdmd v")
    r = run("-h")
    assert r.returncode == 0 and r.stdout.splitlines()[0] == "Usage: tdmd_standalone [options]"
    for flag in ("--data", "--nsteps", "--dt", "--morse", "--eam", "--skin", "--thermo",
                 "--dump-forces", "--dump-final", "--rebuild-every"):
        assert f"  {flag} " in r.stdout
    r = run()
    assert r.returncode == 0 and "Use --data <file> to run a simulation." in r.stdout
    r = run("--data", "x.data", "--morse", "1,2,3")
    assert r.returncode == 1 and "Error: --morse expects D,alpha,r0,rc" in r.stderr
    r = run("--data", os.path.join(ROOT, "no_such_file.data"))
    assert r.returncode == 1 and r.stderr.startswith("Error:")
