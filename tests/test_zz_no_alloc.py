"""tdmd_morse_compute_noalloc (fixed device scratch, no allocation) against
tdmd_morse_compute on the same inputs, called twice in a row, through the C
ABI.  Both run the same kernels with the same launch shape and a fixed-order
reduction, so they agree to 1e-12 relative (forces by the RMS force,
energy and virial componentwise); the file sorts last so the check also
runs after every other GPU test in one process.

The no-allocation claim itself is checked on the device's current CUDA
memory pool (the one stream-ordered allocations draw on), read through the
driver API: its in-use high watermark must not rise over a run of calls and
its reserved size must not change, while tdmd_morse_compute on the same
inputs does raise the watermark (the control)."""
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
    if name == "fcc_64x64x32":  # exactly TDMD_MORSE_NOALLOC_MAX_ATOMS atoms
        a = 3.615
        pos = W.fcc_lattice(64, 64, 32, a)
        rng = np.random.default_rng(11)
        pos += rng.uniform(-0.01, 0.01, size=pos.shape)
        hi = (64 * a, 64 * a, 32 * a)
        pos = np.mod(pos, np.array(hi))
        return pos, (0.0, 0.0, 0.0), hi, g["morse"], g["skin"]
    ncell = {"fcc_55k": 24, "fcc_500k": 50}[name]
    s = W.fcc_system(ncell, 3.615, 300.0, seed=7)
    return s.positions, s.lo, s.hi, g["morse"], g["skin"]


class _Pool:
    """The current memory pool of device 0 through the CUDA driver API."""
    RESERVED_MEM_CURRENT = 5
    USED_MEM_CURRENT = 7
    USED_MEM_HIGH = 8

    def __init__(self):
        self.cu = C.CDLL("libcuda.so.1")
        dev = C.c_int()
        assert self.cu.cuDeviceGet(C.byref(dev), 0) == 0
        self.pool = C.c_void_p()
        assert self.cu.cuDeviceGetMemPool(C.byref(self.pool), dev) == 0

    def get(self, attr):
        v = C.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, C.byref(v)) == 0
        return v.value

    def reset_high(self):
        v = C.c_uint64(0)
        assert self.cu.cuMemPoolSetAttribute(self.pool, self.USED_MEM_HIGH, C.byref(v)) == 0


def _launch(fn, d, nl, n, box, params, precision, f, e, w):
    from tdmd_claude_b200 import _lib
    from tdmd_claude_b200.api import PRECISIONS
    _lib.call(fn, C.c_void_p(d.data_ptr()), C.c_void_p(f.data_ptr()), PRECISIONS[precision],
              C.c_void_p(int(nl.d_neighbors())), C.c_void_p(int(nl.d_offsets())),
              C.c_void_p(int(nl.d_counts())), n, C.byref(box), C.byref(params),
              C.c_void_p(e.data_ptr()), C.c_void_p(w.data_ptr()), None)


def _outputs(torch, n, precision):
    fdt = torch.float64 if precision == "fp64" else torch.float32
    f = torch.full((n, 3), 7.0, dtype=fdt, device="cuda")  # stored, not added
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    w = torch.zeros(6, dtype=torch.float64, device="cuda")
    return f, e, w


def _call(torch, fn, d, nl, n, box, params, precision):
    f, e, w = _outputs(torch, n, precision)
    _launch(fn, d, nl, n, box, params, precision, f, e, w)
    torch.cuda.synchronize()
    return f.double().cpu().numpy(), float(e.item()), w.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["morse_256", "fcc_55k", "fcc_500k", "fcc_64x64x32"])
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


def test_noalloc_allocates_nothing(cuda):
    torch = cuda
    from tdmd_claude_b200 import Box, DeviceNeighborList, MorseParams
    pos, lo, hi, morse, skin = _system("fcc_55k")
    n = len(pos)
    box = Box.make(lo, hi)
    params = MorseParams.make(*morse)
    d = torch.as_tensor(np.ascontiguousarray(pos), dtype=torch.float64, device="cuda")
    nl = DeviceNeighborList()
    nl.build(d, n, box, morse[3], skin)
    # outputs made before the measured region, so nothing in it allocates
    # but the calls themselves
    outs = {p: _outputs(torch, n, p) for p in ("fp64", "mixed")}
    # the first call with an energy does the one-time scratch look-up
    _launch("tdmd_morse_compute_noalloc", d, nl, n, box, params, "mixed", *outs["mixed"])
    pool = _Pool()
    torch.cuda.synchronize()
    pool.reset_high()
    used0 = pool.get(pool.USED_MEM_CURRENT)
    reserved0 = pool.get(pool.RESERVED_MEM_CURRENT)
    for prec in ("fp64", "mixed", "fp64"):
        _launch("tdmd_morse_compute_noalloc", d, nl, n, box, params, prec, *outs[prec])
    torch.cuda.synchronize()
    assert pool.get(pool.USED_MEM_HIGH) <= used0
    assert pool.get(pool.RESERVED_MEM_CURRENT) == reserved0
    # control: the allocating entry point draws its partials from this pool
    pool.reset_high()
    used1 = pool.get(pool.USED_MEM_CURRENT)
    _launch("tdmd_morse_compute", d, nl, n, box, params, "mixed", *outs["mixed"])
    torch.cuda.synchronize()
    assert pool.get(pool.USED_MEM_HIGH) > used1


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
