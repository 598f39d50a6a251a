"""tdmd_morse_compute_noalloc (fixed device scratch, no allocation) against
tdmd_morse_compute on the same inputs, called twice in a row, through the C
ABI.  Both run the same kernels with the same launch shape and a fixed-order
reduction, so they agree to 1e-12 relative (forces by the RMS force,
energy and virial componentwise); the file sorts last so the check also
runs after every other GPU test in one process."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import golden, rel_rms

pytestmark = pytest.mark.gpu

TOL = 1e-12
MAX_ATOMS = 524288  # TDMD_MORSE_NOALLOC_MAX_ATOMS


def _system(name):
    from tdmd_claude_b200 import workloads as W
    g = golden("ref_morse_256.json")
    if name == "morse_256":
        return np.array(g["positions"]), g["lo"], g["hi"], g["morse"], g["skin"]
    ncell = {"fcc_55k": 24, "fcc_500k": 50}[name]
    s = W.fcc_system(ncell, 3.615, 300.0, seed=7)
    return s.positions, s.lo, s.hi, g["morse"], g["skin"]


def _call(torch, fn, d, nl, n, box, params, precision):
    from tdmd_claude_b200 import _lib
    from tdmd_claude_b200.api import PRECISIONS
    fdt = torch.float64 if precision == "fp64" else torch.float32
    f = torch.full((n, 3), 7.0, dtype=fdt, device="cuda")  # stored, not added
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    w = torch.zeros(6, dtype=torch.float64, device="cuda")
    _lib.call(fn, C.c_void_p(d.data_ptr()), C.c_void_p(f.data_ptr()), PRECISIONS[precision],
              C.c_void_p(int(nl.d_neighbors())), C.c_void_p(int(nl.d_offsets())),
              C.c_void_p(int(nl.d_counts())), n, C.byref(box), C.byref(params),
              C.c_void_p(e.data_ptr()), C.c_void_p(w.data_ptr()), None)
    torch.cuda.synchronize()
    return f.double().cpu().numpy(), float(e.item()), w.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["morse_256", "fcc_55k", "fcc_500k"])
def test_noalloc_matches_allocating_entry(cuda, name, precision):
    torch = cuda
    from tdmd_claude_b200 import Box, DeviceNeighborList, MorseParams
    pos, lo, hi, morse, skin = _system(name)
    n = len(pos)
    assert n <= MAX_ATOMS
    box = Box.make(lo, hi)
    params = MorseParams.make(*morse)
    d = torch.as_tensor(np.ascontiguousarray(pos), dtype=torch.float64, device="cuda")
    nl = DeviceNeighborList()
    nl.build(d, n, box, morse[3], skin)
    f0, e0, w0 = _call(torch, "tdmd_morse_compute", d, nl, n, box, params, precision)
    for _ in range(2):  # two calls in a row reuse the same scratch
        f1, e1, w1 = _call(torch, "tdmd_morse_compute_noalloc", d, nl, n, box, params, precision)
        assert rel_rms(f1, f0) <= TOL
        assert abs(e1 - e0) <= TOL * abs(e0)
        assert np.all(np.abs(w1 - w0) <= TOL * np.abs(w0).max())


def test_noalloc_rejects_oversize(cuda):
    torch = cuda
    from tdmd_claude_b200 import Box, MorseParams, _lib
    g = golden("ref_morse_256.json")
    box = Box.make(g["lo"], g["hi"])
    params = MorseParams.make(*g["morse"])
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    idx = torch.zeros(8, dtype=torch.int32, device="cuda")
    p, q = C.c_void_p(buf.data_ptr()), C.c_void_p(idx.data_ptr())
    rc = _lib.lib().tdmd_morse_compute_noalloc(p, p, 0, q, q, q, MAX_ATOMS + 1, C.byref(box),
                                               C.byref(params), p, None, None)
    assert rc == 1  # TDMD_ERR_INVALID_ARGUMENT, nothing launched
    assert "TDMD_MORSE_NOALLOC_MAX_ATOMS" in _lib.lib().tdmd_last_error().decode()
