"""GPU cell list and neighbor list vs the oracle: bit-exact (cell assignment,
ID order in cells, per-atom neighbor order), via the C ABI."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _dev(torch, a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _box(lo, hi, periodic=(1, 1, 1)):
    from tdmd_claude_b200 import Box
    return Box.make(lo, hi, periodic)


def _cases():
    from tdmd_claude_b200 import workloads as W
    g = golden("ref_morse_256.json")
    yield "c0_jitter", np.array(g["positions"]), g["lo"], g["hi"], 6.0, 0.3
    m = golden("run0_morse_256.json")
    yield "perfect_lattice", np.array(m["positions"]), m["lo"], m["hi"], 6.0, 1.0
    s = W.fcc_system(10, 3.615, 300.0, seed=5)
    yield "fcc_4000_eam", s.positions, s.lo, s.hi, 5.0, 0.3
    rng = np.random.default_rng(11)
    L = 23.0
    p = rng.uniform(0, L, size=(1500, 3))
    p[1] = (p[0] + [6.3, 0, 0]) % L      # exactly at r_list (excluded: strict <)
    p[2] = (p[0] + [0, 0, 6.3 - 1e-12]) % L
    yield "random_gas", p, (0, 0, 0), (L, L, L), 6.0, 0.3
    # a box that is not cubic and has a 3-cell axis
    q = rng.uniform(0, 1, size=(900, 3)) * [16.0, 30.0, 41.0] + [-3.0, 2.0, 5.0]
    yield "orthorhombic", q, (-3.0, 2.0, 5.0), (13.0, 32.0, 46.0), 5.0, 0.5
    # a dense blob in a dilute gas: the mean occupancy sizes the shared-memory
    # stage for ~100 candidates, the blob's cells have ~1000, so their rows
    # come from records made on the fly
    blob = rng.uniform(23.0, 37.0, size=(1000, 3))
    gas = rng.uniform(0.0, 60.0, size=(300, 3))
    yield "dense_blob", np.concatenate([blob, gas]), (0, 0, 0), (60, 60, 60), 5.0, 0.3


@pytest.mark.parametrize("case", list(range(6)))
def test_cell_list_bit_exact(cuda, oracle, case):
    from tdmd_claude_b200 import DeviceCellList
    name, pos, lo, hi, rc, skin = list(_cases())[case]
    cl = DeviceCellList()
    d = _dev(cuda, pos, cuda.float64)
    cl.build(d, len(pos), _box(lo, hi), rc + skin)
    nc, atoms, offs, cnts, acell = cl.arrays()
    enc, ecc, eco, eca, eac = oracle.cell_list(pos, lo, hi, rc + skin)
    assert np.array_equal(nc, enc), name
    assert np.array_equal(cnts, ecc), name
    assert np.array_equal(offs, eco), name
    assert np.array_equal(atoms, eca), name
    assert np.array_equal(acell, eac), name


@pytest.mark.parametrize("case", list(range(6)))
def test_full_neighbor_list_bit_exact(cuda, oracle, case):
    from tdmd_claude_b200 import DeviceNeighborList
    name, pos, lo, hi, rc, skin = list(_cases())[case]
    nl = DeviceNeighborList()
    d = _dev(cuda, pos, cuda.float64)
    nl.build(d, len(pos), _box(lo, hi), rc, skin)
    c, o, nb = nl.host_csr()
    ec, eo, enb = oracle.neighbor_list(pos, lo, hi, rc, skin, half=False)
    assert np.array_equal(c, ec), name
    assert np.array_equal(o, eo), name
    assert np.array_equal(nb, enb), name
    assert nl.max_neighbors() == int(ec.max())
    assert nl.total_pairs() == enb.size
    # symmetric: j in list(i) <=> i in list(j)
    pairs = {(i, int(j)) for i in range(len(pos)) for j in nb[o[i]:o[i] + c[i]]}
    assert all((j, i) in pairs for (i, j) in pairs)


def test_neighbor_list_is_twice_the_half_list(cuda, oracle):
    """test_device_neighbor_list.cu:78-128: full-list pairs = 2 x CPU half list."""
    from tdmd_claude_b200 import DeviceNeighborList
    g = golden("ref_morse_256.json")
    pos = np.array(g["positions"])
    nl = DeviceNeighborList()
    nl.build(_dev(cuda, pos, cuda.float64), 256, _box(g["lo"], g["hi"]), 6.0, 0.3)
    assert nl.total_pairs() == 2 * g["half_list"]["total"]


def test_empty_and_single_atom(cuda):
    from tdmd_claude_b200 import DeviceNeighborList
    nl = DeviceNeighborList()
    nl.build(_dev(cuda, np.zeros((1, 3)), cuda.float64), 0, _box((0, 0, 0), (10, 10, 10)), 3.0, 0.3)
    assert nl.total_pairs() == 0
    nl.build(_dev(cuda, np.full((1, 3), 5.0), cuda.float64), 1, _box((0, 0, 0), (10, 10, 10)), 3.0,
             0.3)
    c, o, nb = nl.host_csr()
    assert c.tolist() == [0] and nb.size == 0


def test_invalid_arguments_raise(cuda):
    from tdmd_claude_b200 import DeviceNeighborList, TdmdError
    nl = DeviceNeighborList()
    d = _dev(cuda, np.zeros((4, 3)), cuda.float64)
    with pytest.raises(TdmdError):
        nl.build(d, 4, _box((0, 0, 0), (10, 10, 10)), -1.0, 0.3)
    with pytest.raises(TdmdError):
        nl.build(d, 4, _box((0, 0, 0), (0, 10, 10)), 3.0, 0.3)
