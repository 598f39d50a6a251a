"""A C++ program written against the reference's names (include/tdmd_b200.hpp:
FastPipelineScheduler, DeviceNeighborList, compute_morse_gpu) reproduces the
Python-API results bit for bit in both precision builds."""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def rd_(precision):
    """The mixed build's `real` is float: its dt, skin, masses and Morse
    parameters arrive rounded to float."""
    return (lambda x: float(np.float32(x))) if precision == "mixed" else float  # noqa: E731


@pytest.mark.parametrize("define,precision", [("TDMD_PRECISION_FP64", "fp64"),
                                              ("TDMD_PRECISION_MIXED", "mixed")])
def test_cpp_layer_runs_gpu_path(cuda, tmp_path, define, precision):
    torch = cuda
    from tdmd_claude_b200 import (Box, DeviceNeighborList, FastPipelineScheduler, MorseParams,
                                  _lib, compute_morse_gpu, make_config)
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "wrapper_gpu")
    subprocess.run([gxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", f"-D{define}",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA_HOME, "include"),
                    os.path.join(ROOT, "tests", "cpp", "wrapper_gpu.cpp"), "-o", exe, _lib.LIB_PATH,
                    f"-Wl,-rpath,{os.path.dirname(_lib.LIB_PATH)}",
                    "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart"],
                   check=True, capture_output=True, text=True)
    g = golden("ref_morse_256.json")
    pos, vel = np.array(g["positions"]), np.array(g["velocities"])
    n, lo, hi = len(pos), g["lo"][0], g["hi"][0]
    inp, outp = str(tmp_path / "in.txt"), str(tmp_path / "out.txt")
    with open(inp, "w") as f:
        f.write(f"{n} {lo!r} {hi!r}\n")
        for p, v in zip(pos, vel):
            f.write(" ".join(repr(float(x)) for x in (*p, *v)) + "\n")
    r = subprocess.run([exe, inp, outp], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rows = open(outp).read().split("\n")
    sched_rows = np.array([[float(x) for x in l.split()] for l in rows[:n]])
    e_cpp = float(rows[n])
    f_cpp = np.array([[float(x) for x in l.split()] for l in rows[n + 1:2 * n + 1]])
    cells = rows[2 * n + 1].split()
    # zone calls: two zones = the whole system; the zone kick moved its zone only
    ez, dfz, vlo, vhi = (float(x) for x in rows[2 * n + 2].split())
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert abs(ez - e_cpp) <= tol * abs(e_cpp)
    assert dfz <= tol * np.abs(f_cpp).max()
    assert vlo == 0.0 and vhi > 0.0
    L = hi - lo
    nc = max(3, int(np.floor(L / (6.0 + rd_(precision)(0.3)))))
    assert [int(x) for x in cells[:3]] == [nc] * 3
    assert [float(x) for x in cells[3:]] == [L / nc] * 3
    # the same through the Python API
    rd = rd_(precision)
    box = Box.make((lo,) * 3, (hi,) * 3)
    mp = MorseParams.make(rd(0.3429), rd(1.3588), rd(2.866), 6.0)
    s = FastPipelineScheduler(box, n, mp, make_config(dt=rd(0.001), r_skin=rd(0.3),
                                                      rebuild_every=10, precision=precision,
                                                      lanes_per_atom=4))
    s.upload(pos, vel, None, np.ones(n, np.int32), np.arange(1, n + 1, dtype=np.int32),
             np.array([1.0, rd(63.546)]))
    s.run_until(20)
    st = s.download()
    assert np.array_equal(sched_rows[:, 0:3], st.positions)
    assert np.array_equal(sched_rows[:, 3:6], st.velocities)
    assert np.array_equal(sched_rows[:, 6:9], st.forces.astype(np.float64))
    d = torch.as_tensor(st.positions, dtype=torch.float64, device="cuda")
    nl = DeviceNeighborList()
    nl.build(d, n, box, 6.0, rd(0.3))
    fdt = torch.float64 if precision == "fp64" else torch.float32
    f = torch.zeros((n, 3), dtype=fdt, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    compute_morse_gpu(d, f, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box, mp, e,
                      precision=precision)
    torch.cuda.synchronize()
    assert e_cpp == float(e.item())
    assert np.array_equal(f_cpp, f.double().cpu().numpy())
    _ = C
