"""The oracle's force-matching gradients (FP64 restatement of the adjoint)
against central finite differences of its own loss (h = 1e-6 relative).
Morse: all three parameters.  EAM: sampled coefficients of every spline
(F, rho, phi), single-element and ternary tables; the error is measured
against the largest gradient entry of that spline, since entries near zero
are dominated by round-off in the difference quotient."""
from __future__ import annotations

import numpy as np

MORSE = (0.3429, 1.3588, 2.866, 5.0)


def _snapshots(ntypes, rng):
    from tdmd_claude_b200 import workloads as W
    ss = [W.fcc_system(3, 3.615, 1200.0, s, jitter=0.1,
                       types=rng.integers(1, ntypes + 1, size=108).astype(np.int32),
                       masses=(63.5,) * ntypes) for s in (1, 2)]
    return (np.stack([s.positions for s in ss]), np.stack([s.types for s in ss]), ss[0].lo,
            ss[0].hi)


def test_morse_gradient_matches_finite_differences(oracle):
    rng = np.random.default_rng(5)
    pos, _, lo, hi = _snapshots(1, rng)
    tgt = rng.normal(0.0, 0.3, size=pos.shape)
    p = np.array(MORSE[:3])
    _, g = oracle.morse_fm_loss_grad(pos, lo, hi, *p, MORSE[3], tgt)
    for k in range(3):
        h = 1e-6 * p[k]
        up, dn = p.copy(), p.copy()
        up[k] += h
        dn[k] -= h
        fd = (oracle.morse_fm_loss_grad(pos, lo, hi, *up, MORSE[3], tgt)[0] -
              oracle.morse_fm_loss_grad(pos, lo, hi, *dn, MORSE[3], tgt)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * abs(g[k])


def _eam_case(tables, ntypes, oracle, seed):
    rng = np.random.default_rng(seed)
    pos, types, lo, hi = _snapshots(ntypes, rng)
    t = tables
    e = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    tgt = rng.normal(0.0, 0.3, size=pos.shape)
    _, gF, gr, gp = e.fm_loss_grad(pos, types, lo, hi, tgt)
    worst = 0.0
    for kind, g in ((0, gF), (1, gr), (2, gp)):
        for sp in range(g.shape[0]):
            scale = np.abs(g[sp]).max()
            assert scale > 0.0
            nz = np.nonzero(np.abs(g[sp]) > 1e-8 * scale)[0]
            for k in rng.choice(nz, size=min(4, len(nz)), replace=False):
                base = e.coeffs(kind, sp).copy()
                h = 1e-6 * max(abs(base[k]), 1e-3)
                up, dn = base.copy(), base.copy()
                up[k] += h
                dn[k] -= h
                e.set_coeffs(kind, sp, up)
                lp = e.fm_loss_grad(pos, types, lo, hi, tgt)[0]
                e.set_coeffs(kind, sp, dn)
                lm = e.fm_loss_grad(pos, types, lo, hi, tgt)[0]
                e.set_coeffs(kind, sp, base)
                worst = max(worst, abs((lp - lm) / (2 * h) - g[sp][k]) / scale)
    return worst


def test_eam_gradient_matches_finite_differences(oracle):
    from tdmd_claude_b200 import workloads as W
    assert _eam_case(W.cu_eam_tables(), 1, oracle, 5) < 1e-5
    assert _eam_case(W.ternary_eam_tables(), 3, oracle, 6) < 1e-5
