"""The ID-ordered energy mode (tdmd_set_deterministic_reduce) against the
reference's own deterministic build: the reference's GPU path compiled from
its sources with -DTDMD_PRECISION_FP64=1 -DTDMD_DETERMINISTIC_REDUCE=1
(oracle/_ref/libtdmd_ref_gpu_fp64_det.so), its DeviceNeighborList and
compute_morse_gpu / DeviceEam::compute (src/potentials/device_morse.cu:
16-30,136-170; device_eam.cu:20,342-418; ADR 0010).  On the same positions
both give the same neighbor rows (bit-exact lists), and in this mode the
same per-atom arithmetic and the same one-thread ID-ordered sums: energies
and forces are compared for bit equality, and two calls in a row give the
same bits.  The default mode agrees to 1e-12 relative."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, golden, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refdet():
    p = os.path.join(ROOT, "oracle", "_ref", "libtdmd_ref_gpu_fp64_det.so")
    if not os.path.exists(p):
        pytest.skip("the reference's deterministic FP64 build was not built (make -C oracle refgpu)")
    L = C.CDLL(p)
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
    L.refgpu_last_error.restype = C.c_char_p
    L.refgpu_morse_forces.argtypes = [f64p, C.c_int32, f64p, f64p, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double, f64p,
                                      C.POINTER(C.c_double)]
    L.refgpu_morse_forces.restype = C.c_int32
    L.refgpu_eam_forces.argtypes = [C.c_char_p, f64p, i32p, C.c_int32, f64p, f64p, C.c_double,
                                    f64p, C.POINTER(C.c_double)]
    L.refgpu_eam_forces.restype = C.c_int32
    return L


@pytest.fixture
def det_mode():
    from tdmd_claude_b200 import deterministic_reduce, set_deterministic_reduce
    assert not deterministic_reduce()
    set_deterministic_reduce(True)
    yield
    set_deterministic_reduce(False)


def _ours_morse(torch, pos, lo, hi, morse, skin):
    from tdmd_claude_b200 import Box, DeviceNeighborList, MorseParams, compute_morse_gpu
    n = len(pos)
    d = torch.as_tensor(np.ascontiguousarray(pos), dtype=torch.float64, device="cuda")
    box = Box.make(lo, hi)
    nl = DeviceNeighborList()
    nl.build(d, n, box, morse[3], skin)
    out = []
    for _ in range(2):
        f = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        compute_morse_gpu(d, f, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box,
                          MorseParams.make(*morse), e)
        torch.cuda.synchronize()
        out.append((float(e.item()), f.cpu().numpy()))
    return out


def _ours_eam(torch, eam, pos, types, lo, hi, skin):
    from tdmd_claude_b200 import Box, DeviceEam, DeviceNeighborList
    n = len(pos)
    d = torch.as_tensor(np.ascontiguousarray(pos), dtype=torch.float64, device="cuda")
    t = torch.as_tensor(np.ascontiguousarray(types, np.int32), device="cuda")
    box = Box.make(lo, hi)
    nl = DeviceNeighborList()
    nl.build(d, n, box, eam.cutoff(), skin)
    de = DeviceEam()
    de.upload_tables(eam)
    out = []
    for _ in range(2):
        f = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        de.compute(d, f, t, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box, e)
        torch.cuda.synchronize()
        out.append((float(e.item()), f.cpu().numpy()))
    return out


def _morse_cases():
    g = golden("ref_morse_256.json")
    yield "c0_jitter", np.array(g["positions"]), g["lo"], g["hi"], g["morse"], g["skin"]
    m = golden("run0_morse_256.json")
    yield "run0_lattice", np.array(m["positions"]), m["lo"], m["hi"], m["morse"], m["skin"]
    from tdmd_claude_b200 import workloads as W
    s = W.fcc_system(10, 3.615, 300.0, seed=8)
    yield "fcc_4000", s.positions, s.lo, s.hi, g["morse"], 0.3


@pytest.mark.parametrize("case", [0, 1, 2])
def test_morse_energy_bits_equal_reference_deterministic_build(cuda, refdet, det_mode, case):
    name, pos, lo, hi, morse, skin = list(_morse_cases())[case]
    n = len(pos)
    f_ref = np.zeros((n, 3))
    e_ref = C.c_double()
    assert refdet.refgpu_morse_forces(np.ascontiguousarray(pos), n, np.array(lo, float),
                                      np.array(hi, float), *morse, skin, f_ref,
                                      C.byref(e_ref)) == 0, refdet.refgpu_last_error()
    (e1, f1), (e2, f2) = _ours_morse(cuda, pos, lo, hi, morse, skin)
    assert e1 == e_ref.value, (name, e1, e_ref.value)
    assert np.array_equal(f1, f_ref), name
    assert e2 == e1 and np.array_equal(f2, f1)


def _eam_cases(mishin_setfl, tmp):
    from tdmd_claude_b200 import io as TIO
    from tdmd_claude_b200 import workloads as W
    m = golden("run0_morse_256.json")
    yield "mishin_256", mishin_setfl, np.array(m["positions"]), np.ones(256, np.int32), \
        m["lo"], m["hi"], 1.0
    p = os.path.join(tmp, "cu.eam.alloy")
    TIO.write_setfl(p, W.cu_eam_tables())
    s = W.fcc_system(10, 3.615, 300.0, seed=9)
    yield "analytic_4000", p, s.positions, s.types, s.lo, s.hi, 0.3
    p3 = os.path.join(tmp, "ternary.eam.alloy")
    TIO.write_setfl(p3, W.ternary_eam_tables())
    t = W.ternary(6, seed=4)
    yield "ternary_864", p3, t.positions, t.types, t.lo, t.hi, 0.3


@pytest.mark.parametrize("case", [0, 1, 2])
def test_eam_energy_bits_equal_reference_deterministic_build(cuda, refdet, det_mode,
                                                             mishin_setfl, tmp_path, case):
    from tdmd_claude_b200 import EamAlloy
    name, setfl, pos, types, lo, hi, skin = list(_eam_cases(mishin_setfl, str(tmp_path)))[case]
    n = len(pos)
    f_ref = np.zeros((n, 3))
    e_ref = C.c_double()
    assert refdet.refgpu_eam_forces(setfl.encode(), np.ascontiguousarray(pos),
                                    np.ascontiguousarray(types, np.int32), n,
                                    np.array(lo, float), np.array(hi, float), skin, f_ref,
                                    C.byref(e_ref)) == 0, refdet.refgpu_last_error()
    eam = EamAlloy().read_setfl(setfl)
    (e1, f1), (e2, f2) = _ours_eam(cuda, eam, pos, types, lo, hi, skin)
    assert e1 == e_ref.value, (name, e1, e_ref.value)
    assert np.array_equal(f1, f_ref), name
    assert e2 == e1 and np.array_equal(f2, f1)


def test_default_mode_agrees_with_deterministic_mode(cuda, mishin_setfl):
    """Jittered positions (on the perfect lattice the forces are rounding
    noise of ~1e-15 and no relative comparison means anything)."""
    from tdmd_claude_b200 import EamAlloy, set_deterministic_reduce
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    eam = EamAlloy().read_setfl(mishin_setfl)
    base = _ours_eam(cuda, eam, pos, np.ones(256, np.int32), g["lo"], g["hi"], 0.3)[0]
    set_deterministic_reduce(True)
    try:
        det = _ours_eam(cuda, eam, pos, np.ones(256, np.int32), g["lo"], g["hi"], 0.3)[0]
    finally:
        set_deterministic_reduce(False)
    assert abs(base[0] - det[0]) <= 1e-12 * abs(det[0])
    assert rel_rms(base[1], det[1]) <= 1e-12
