"""Shared fixtures.  `-m gpu` tests need a CUDA device and the in-tree
libtdmd_b200.so; everything else runs on the CPU."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.oracle import reference_tree  # noqa: E402

REF_TREE = reference_tree()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running")


def golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def ref_lib(oracle):
    """The reference's own CPU path (skips where it was not built)."""
    R = oracle.ref()
    if R is None:
        pytest.skip("reference CPU path not built (oracle/_ref)")
    return R


def golden_file(name: str, tmp_dir: str) -> str:
    """Path of a golden fixture; a `.xz` one is decompressed into tmp_dir."""
    import lzma
    src = os.path.join(GOLDEN, name)
    if not name.endswith(".xz"):
        return src
    dst = os.path.join(tmp_dir, name[:-3])
    if not os.path.exists(dst):
        with lzma.open(src, "rb") as f, open(dst, "wb") as o:
            o.write(f.read())
    return dst


@pytest.fixture(scope="session")
def mishin_setfl(tmp_path_factory):
    """The reference's Mishin Cu setfl (tests/data/Cu_mishin1.eam.alloy)."""
    g = golden("run0_eam_256.json")
    return golden_file(g["potential_file"], str(tmp_path_factory.mktemp("golden")))


def reference_file(rel: str) -> str:
    if REF_TREE is None:
        pytest.skip(f"reference tree not found (set TDMD_REFERENCE_TREE); {rel} unavailable")
    p = os.path.join(REF_TREE, rel)
    if not os.path.exists(p):
        pytest.skip(f"reference file {rel} not available here")
    return p


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tdmd_claude_b200 import _lib
    _lib.lib()
    return torch


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def two_element_tables():
    """Two elements, every function distinct: F_A = -sqrt(rho),
    F_B = -1.7 sqrt(rho); f_A = exp(-1.1 r), f_B = 2.5 exp(-0.7 r);
    r phi_AA = 0.4 exp(-2.1 r), r phi_AB = 0.9 exp(-1.95 r),
    r phi_BB = 1.3 exp(-1.75 r); grids drho 0.01 x 500, dr 0.012 x 501
    (cutoff 6.0)."""
    from tdmd_claude_b200 import workloads as W
    nrho, drho, nr, dr = 500, 0.01, 501, 0.012
    rg = np.arange(nrho) * drho
    r = np.arange(nr) * dr
    F = np.stack([-np.sqrt(rg), -1.7 * np.sqrt(rg)])
    rho = np.stack([np.exp(-1.1 * r), 2.5 * np.exp(-0.7 * r)])
    rphi = np.stack([0.4 * np.exp(-2.1 * r), 0.9 * np.exp(-1.95 * r), 1.3 * np.exp(-1.75 * r)])
    return W.EamTables(2, nrho, drho, nr, dr, 6.0, F, rho, rphi, ("A", "B"), (10.0, 20.0))
