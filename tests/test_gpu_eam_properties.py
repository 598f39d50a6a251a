"""Physical and bookkeeping properties of the GPU EAM and Morse paths, the
ones the reference's unit tests state (tests/unit/test_eam.cpp,
tests/unit/test_morse.cpp), checked here on inputs this suite generates:

* two atoms at the FCC nearest-neighbor distance: bound, equal and
  opposite, nonzero forces (test_eam.cpp:32-67);
* a two-element alloy whose six functions all differ: swapping the type
  labels must change energy and forces, the same labels must give the same
  bits, and the GPU must agree with the oracle (test_eam.cpp:163-290);
* per-atom densities equal an O(N^2) brute-force sum (test_eam.cpp:313-395);
* Morse energy and force against the closed form over a radius sweep that
  crosses the cutoff (test_morse.cpp:39-78).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _box(lo, hi):
    from tdmd_claude_b200 import Box
    return Box.make(lo, hi)


def _eam(torch, eam, pos, types, lo, hi, skin, precision):
    """DeviceNeighborList + DeviceEam.compute: forces, PE, rho."""
    from tdmd_claude_b200 import DeviceEam, DeviceNeighborList
    n = len(pos)
    box = _box(lo, hi)
    d = torch.as_tensor(np.ascontiguousarray(pos), dtype=torch.float64, device="cuda")
    t = torch.as_tensor(np.ascontiguousarray(types), dtype=torch.int32, device="cuda")
    nl = DeviceNeighborList()
    nl.build(d, n, box, eam.cutoff(), skin)
    de = DeviceEam()
    de.upload_tables(eam)
    fdt = torch.float64 if precision == "fp64" else torch.float32
    f = torch.zeros((n, 3), dtype=fdt, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    w = torch.zeros(6, dtype=torch.float64, device="cuda")
    rho = torch.zeros(n, dtype=torch.float64, device="cuda")
    fp = torch.zeros(n, dtype=torch.float64, device="cuda")
    de.compute(d, f, t, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n, box, e, w, rho, fp,
               precision=precision)
    torch.cuda.synchronize()
    return f.double().cpu().numpy(), float(e.item()), rho.cpu().numpy()


def _tables_eam(t):
    from tdmd_claude_b200 import EamAlloy
    return EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho,
                                t.rphi)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_two_atoms(cuda, oracle, precision):
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables()
    pos = np.array([[8.0, 10.0, 10.0], [10.556, 10.0, 10.0]])
    types = np.ones(2, np.int32)
    f, e, _ = _eam(cuda, _tables_eam(t), pos, types, (0, 0, 0), (20, 20, 20), 0.5, precision)
    assert e < 0.0
    assert np.abs(f[0] + f[1]).max() < 1e-10
    assert abs(f[0, 0]) > 1e-6
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    r = oe.forces(pos, types, (0, 0, 0), (20, 20, 20), 0.5)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.abs(f - r["forces"]).max() <= tol * np.abs(r["forces"]).max()
    assert abs(e - r["pe"]) <= tol * abs(r["pe"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_type_labels_matter(cuda, oracle, precision):
    import os
    import tempfile

    from conftest import two_element_tables

    from tdmd_claude_b200 import EamAlloy
    from tdmd_claude_b200 import io as TIO
    t = two_element_tables()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "ab.eam.alloy")
        TIO.write_setfl(p, t, comment="two-element test alloy")
        eam = EamAlloy().read_setfl(p)
    assert eam.ntypes() == 2 and abs(eam.cutoff() - 6.0) < 1e-12
    pos = np.array([[3.0, 8.0, 8.0], [5.4, 8.0, 8.0], [6.9, 6.2, 8.0], [6.6, 8.3, 9.9]])
    lo, hi, skin = (0, 0, 0), (16, 16, 16), 0.5
    ab = np.array([1, 2, 1, 2], np.int32)
    ba = np.array([2, 1, 2, 1], np.int32)
    fa, ea, _ = _eam(cuda, eam, pos, ab, lo, hi, skin, precision)
    fb, eb, _ = _eam(cuda, eam, pos, ba, lo, hi, skin, precision)
    assert abs(ea - eb) > 1e-3
    assert np.abs(fa - fb).max() > 1e-3
    fa2, ea2, _ = _eam(cuda, eam, pos, ab, lo, hi, skin, precision)
    assert ea2 == ea and np.array_equal(fa2, fa)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    tol = 1e-10 if precision == "fp64" else 1e-5
    for types, f, e in ((ab, fa, ea), (ba, fb, eb)):
        r = oe.forces(pos, types, lo, hi, skin)
        assert np.abs(f - r["forces"]).max() <= tol * np.abs(r["forces"]).max()
        assert abs(e - r["pe"]) <= tol * abs(r["pe"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eam_density_equals_brute_force(cuda, precision):
    """rho_i from the neighbor-list pass against a sum over all atom pairs
    (minimum image, r < cutoff) with the same spline rows, in FP64."""
    from conftest import golden

    from tdmd_claude_b200 import workloads as W
    m = golden("ref_morse_256.json")
    pos = np.array(m["positions"])
    lo, hi = np.array(m["lo"], float), np.array(m["hi"], float)
    t = W.cu_eam_tables()
    eam = _tables_eam(t)
    n = len(pos)
    _, _, rho = _eam(cuda, eam, pos, np.ones(n, np.int32), lo, hi, 0.3, precision)
    c = eam.coeffs(1, 0)
    k = t.nr - 1
    a, b, cc, dd = c[:k], c[k:2 * k], c[2 * k:3 * k], c[3 * k:]
    L = hi - lo
    d = pos[None, :, :] - pos[:, None, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d * d).sum(-1))
    mask = (r < t.cutoff) & ~np.eye(n, dtype=bool)
    rr = r[mask]
    idx = np.clip((rr / t.dr).astype(np.int64), 0, t.nr - 2)
    x = rr - idx * t.dr
    val = a[idx] + x * (b[idx] + x * (cc[idx] + x * dd[idx]))
    brute = np.zeros(n)
    np.add.at(brute, np.nonzero(mask)[0], val)
    assert np.all(rho > 0.01)
    tol = 1e-10 if precision == "fp64" else 1e-5
    assert np.abs(rho - brute).max() <= tol * np.abs(brute).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_morse_closed_form_sweep(cuda, precision):
    """U(r) = D((1 - e)^2 - 1), e = exp(-alpha (r - r0)), and the force
    dU/dr = 2 D alpha (1 - e) e on atom 0 along +x, for r = 2.0 ... 8.5
    in steps of 0.5 (rc = 6.0): zero at and beyond the cutoff.  The mixed
    path decides r < rc in FP32, so its sweep leaves out r = rc itself."""
    from tdmd_claude_b200 import DeviceNeighborList, MorseParams, compute_morse_gpu
    import torch
    D, al, r0, rc = 0.3429, 1.3588, 2.866, 6.0
    for r in np.arange(2.0, 9.0, 0.5):
        if precision == "mixed" and r == rc:
            continue
        pos = np.array([[10.0, 15.0, 15.0], [10.0 + r, 15.0, 15.0]])
        d = torch.as_tensor(pos, dtype=torch.float64, device="cuda")
        box = _box((0, 0, 0), (30, 30, 30))
        nl = DeviceNeighborList()
        nl.build(d, 2, box, rc, 0.3)
        fdt = torch.float64 if precision == "fp64" else torch.float32
        f = torch.zeros((2, 3), dtype=fdt, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        compute_morse_gpu(d, f, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), 2, box,
                          MorseParams.make(D, al, r0, rc), e, None, precision=precision)
        torch.cuda.synchronize()
        f = f.double().cpu().numpy()
        ex = np.exp(-al * (r - r0))
        u = D * ((1 - ex) ** 2 - 1) if r < rc else 0.0
        dudr = 2 * D * al * (1 - ex) * ex if r < rc else 0.0
        if precision == "fp64":
            assert abs(float(e.item()) - u) <= 1e-12 * max(1.0, abs(u)), r
            assert abs(f[0, 0] - dudr) <= 1e-12 * max(1.0, abs(dudr)), r
        else:
            assert abs(float(e.item()) - u) <= 1e-6 + 1e-5 * abs(u), r
            assert abs(f[0, 0] - dudr) <= 1e-6 + 1e-5 * abs(dudr), r
        assert f[0, 0] == -f[1, 0] and np.all(f[:, 1:] == 0.0), r
