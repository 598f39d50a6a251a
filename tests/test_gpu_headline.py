"""Parity at the benchmarked configurations, GPU against the oracle.

* The bench's headline system: 32^3 Cu FCC cells = 131 072 atoms (seed
  4321, +-0.01 A jitter, 300 K), the analytic EAM tabulated as setfl
  splines (rc 5.0), skin 0.3, rebuild every 10 steps, launch shapes from the
  autotuner as in the bench.  The scheduler's own neighbor list (cell-ordered
  atoms, a list stage sized from the upload's largest cell) and the
  free-function cell/neighbor lists are bit-exact to the oracle
  (test_device_neighbor_list.cu:16-128); FP64 forces, energy and virial
  agree to 1e-10 relative (test_device_eam.cu:24-92 with the FP64
  tolerance); mixed forces to 1e-5 RMS relative and energy to 1e-6, against
  the oracle's FP64 values, not this library's FP64 path.  A 10-step
  window (the fused kick + drift of the mixed path) and the next step (the
  first rebuild) follow the oracle's scheduler loop.
* An equiatomic random ternary, 20^3 cells = 32 000 atoms, with the
  three-species analytic EAM of the 4 M-atom workload: the same checks.

The oracle needs ~0.5 s per 131 072-atom force evaluation (one host core)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu

SKIN = 0.3


def _wrap_diff(a, b, L):
    d = a - b
    return d - np.round(d / L) * L


@pytest.fixture(scope="module")
def headline(oracle):
    from tdmd_claude_b200 import workloads as W
    s = W.fcc_system(32, 3.615, 300.0, 4321)
    t = W.cu_eam_tables()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    ref = oe.forces(s.positions, s.types, s.lo, s.hi, SKIN)
    lists = oracle.neighbor_list(s.positions, s.lo, s.hi, t.cutoff, SKIN, half=False)
    return s, t, oe, ref, lists


@pytest.fixture(scope="module")
def ternary(oracle):
    from tdmd_claude_b200 import workloads as W
    s = W.ternary(20, seed=99)
    t = W.ternary_eam_tables()
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    ref = oe.forces(s.positions, s.types, s.lo, s.hi, SKIN)
    lists = oracle.neighbor_list(s.positions, s.lo, s.hi, t.cutoff, SKIN, half=False)
    return s, t, oe, ref, lists


def _sched(s, t, precision):
    from tdmd_claude_b200 import Box, EamAlloy, FastPipelineScheduler, make_config
    eam = EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    sch = FastPipelineScheduler(Box.make(s.lo, s.hi), s.n, eam,
                                make_config(r_skin=SKIN, precision=precision))
    sch.upload(s.positions, s.velocities, None, s.types, s.ids, s.masses)
    return sch


def _check_lists(sch, lists):
    c, o, nb = sch.neighbor_list()
    ec, eo, enb = lists
    assert np.array_equal(c, ec)
    assert np.array_equal(o, eo)
    assert np.array_equal(nb, enb)


def _check_forces(sch, ref, precision):
    st = sch.download()
    pe, _, w = sch.energies()
    if precision == "fp64":
        assert rel_rms(st.forces, ref["forces"]) <= 1e-10
        assert abs(pe - ref["pe"]) <= 1e-10 * abs(ref["pe"])
        assert np.abs(w - ref["virial"]).max() <= 1e-10 * np.abs(ref["virial"]).max()
    else:
        assert rel_rms(st.forces, ref["forces"]) <= 1e-5
        assert abs(pe - ref["pe"]) <= 1e-6 * abs(ref["pe"])
        assert np.abs(w - ref["virial"]).max() <= 1e-6 * np.abs(ref["virial"]).max()


def test_headline_free_function_lists_bit_exact(cuda, oracle, headline):
    from tdmd_claude_b200 import Box, DeviceCellList, DeviceNeighborList
    s, t, _, _, lists = headline
    d = cuda.as_tensor(s.positions, dtype=cuda.float64, device="cuda")
    box = Box.make(s.lo, s.hi)
    cl = DeviceCellList()
    cl.build(d, s.n, box, t.cutoff + SKIN)
    nc, atoms, offs, cnts, acell = cl.arrays()
    enc, ecc, eco, eca, eac = oracle.cell_list(s.positions, s.lo, s.hi, t.cutoff + SKIN)
    assert np.array_equal(nc, enc) and np.array_equal(cnts, ecc) and np.array_equal(offs, eco)
    assert np.array_equal(atoms, eca) and np.array_equal(acell, eac)
    nl = DeviceNeighborList()
    nl.build(d, s.n, box, t.cutoff, SKIN)
    c, o, nb = nl.host_csr()
    ec, eo, enb = lists
    assert np.array_equal(c, ec) and np.array_equal(o, eo) and np.array_equal(nb, enb)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_headline_scheduler_step0(cuda, headline, precision):
    s, t, _, ref, lists = headline
    sch = _sched(s, t, precision)
    sch.run_until(0)
    _check_lists(sch, lists)
    _check_forces(sch, ref, precision)
    sch.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_headline_scheduler_window(cuda, oracle, headline, precision):
    """One bench window of 10 steps, then the next step, whose drift is
    followed by the first rebuild (maybe_rebuild_nlist: steps since the last
    build reach rebuild_every), against the oracle's restatement of the
    scheduler loop; the rebuilt list equals the oracle's list of the
    scheduler's positions at that step."""
    s, t, oe, _, _ = headline
    sch = _sched(s, t, precision)
    sch.run_until(10)
    sch.run_until(11)
    st = sch.download()
    r = oracle.md_run(s.positions, s.velocities, s.types, s.masses, s.lo, s.hi, 0.001, SKIN, 10,
                      [10, 11], eam=oe)
    L = np.array(s.hi) - np.array(s.lo)
    dx = np.abs(_wrap_diff(st.positions, r["pos"], L)).max()
    if precision == "fp64":
        assert dx < 1e-10
        assert np.abs(st.velocities - r["vel"]).max() < 1e-9
        assert rel_rms(st.forces, r["forces"]) < 1e-9
    else:
        assert dx < 1e-5
        # force error at the mixed path's own positions
        ref = oe.forces(st.positions, s.types, s.lo, s.hi, SKIN)
        assert rel_rms(st.forces, ref["forces"]) <= 1e-5
    _check_lists(sch, oracle.neighbor_list(st.positions, s.lo, s.hi, t.cutoff, SKIN, half=False))
    sch.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ternary_32k_scheduler_step0(cuda, ternary, precision):
    s, t, _, ref, lists = ternary
    assert s.n == 32000 and t.ntypes == 3
    sch = _sched(s, t, precision)
    sch.run_until(0)
    _check_lists(sch, lists)
    _check_forces(sch, ref, precision)
    sch.close()
