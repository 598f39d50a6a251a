"""Force-matching loss and adjoint gradients on the GPU (tdmd_fit_*) against
the oracle's FP64 restatement, central finite differences of the GPU loss,
and the torch.autograd / Adam harness.

Tolerances: FP64 loss 1e-10 relative, gradients 1e-9 of the largest entry
per spline (1e-9 relative for the Morse parameters); mixed (FP32 pair
arithmetic, FP64 accumulation) loss 1e-5, gradients 1e-4 of the largest
entry."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MORSE = (0.3429, 1.3588, 2.866, 5.0)


def _snapshots(ntypes, seed, nsnap=2, ncell=3):
    from tdmd_claude_b200 import workloads as W
    rng = np.random.default_rng(seed)
    n = 4 * ncell ** 3
    ss = [W.fcc_system(ncell, 3.615, 1200.0, seed + s, jitter=0.1,
                       types=rng.integers(1, ntypes + 1, size=n).astype(np.int32),
                       masses=(63.5,) * ntypes) for s in range(nsnap)]
    pos = np.stack([s.positions for s in ss])
    types = np.stack([s.types for s in ss])
    return pos, types, ss[0].lo, ss[0].hi, rng.normal(0.0, 0.3, size=pos.shape)


def _fm(pos, types, lo, hi, precision):
    from tdmd_claude_b200 import Box
    from tdmd_claude_b200.fitting import ForceMatch
    return ForceMatch(pos, types, Box.make(lo, hi), MORSE[3], precision)


def _morse_gpu(fm, torch, p):
    prm = torch.tensor(p, dtype=torch.float64, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    grad = torch.zeros(3, dtype=torch.float64, device="cuda")
    fm.morse(prm, loss, grad)
    torch.cuda.synchronize()
    return float(loss.item()), grad.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_morse_loss_and_gradient_vs_oracle(cuda, oracle, precision):
    torch = cuda
    pos, types, lo, hi, tgt = _snapshots(1, 11)
    fm = _fm(pos, types, lo, hi, precision)
    fm.set_targets(tgt)
    loss, g = _morse_gpu(fm, torch, MORSE[:3])
    lo_, go = oracle.morse_fm_loss_grad(pos, lo, hi, *MORSE, tgt)
    tol_l, tol_g = (1e-10, 1e-9) if precision == "fp64" else (1e-5, 1e-4)
    assert abs(loss - lo_) <= tol_l * lo_
    assert np.all(np.abs(g - go) <= tol_g * np.abs(go))


def test_morse_gradient_matches_gpu_finite_differences(cuda):
    torch = cuda
    pos, types, lo, hi, tgt = _snapshots(1, 12)
    fm = _fm(pos, types, lo, hi, "fp64")
    fm.set_targets(tgt)
    p = np.array(MORSE[:3])
    _, g = _morse_gpu(fm, torch, p)
    for k in range(3):
        h = 1e-6 * p[k]
        up, dn = p.copy(), p.copy()
        up[k] += h
        dn[k] -= h
        fd = (_morse_gpu(fm, torch, up)[0] - _morse_gpu(fm, torch, dn)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * abs(g[k])


def _tables(ntypes):
    from tdmd_claude_b200 import EamAlloy
    from tdmd_claude_b200 import workloads as W
    t = W.cu_eam_tables() if ntypes == 1 else W.ternary_eam_tables()
    return t, EamAlloy.from_tables(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho,
                                   t.rphi)


def _eam_gpu(fm, torch, meta, F, rho, phi):
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    gF, gr, gp = torch.empty_like(F), torch.empty_like(rho), torch.empty_like(phi)
    fm.eam(meta, F, rho, phi, loss, gF, gr, gp)
    torch.cuda.synchronize()
    return float(loss.item()), gF.cpu().numpy(), gr.cpu().numpy(), gp.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("ntypes", [1, 3])
def test_eam_loss_and_gradient_vs_oracle(cuda, oracle, precision, ntypes):
    torch = cuda
    from tdmd_claude_b200.fitting import eam_coeff_tensors, eam_table_meta
    pos, types, lo, hi, tgt = _snapshots(ntypes, 20 + ntypes)
    t, eam = _tables(ntypes)
    fm = _fm(pos, types, lo, hi, precision)
    fm.set_targets(tgt)
    F, rho, phi = eam_coeff_tensors(eam)
    loss, gF, gr, gp = _eam_gpu(fm, torch, eam_table_meta(eam), F, rho, phi)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    lo_, oF, orho, ophi = oe.fm_loss_grad(pos, types, lo, hi, tgt)
    tol_l, tol_g = (1e-10, 1e-9) if precision == "fp64" else (1e-5, 1e-4)
    assert abs(loss - lo_) <= tol_l * lo_
    for got, ref in ((gF, oF), (gr, orho), (gp, ophi)):
        for sp in range(ref.shape[0]):
            assert np.abs(got[sp] - ref[sp]).max() <= tol_g * np.abs(ref[sp]).max()


def test_eam_gradient_matches_gpu_finite_differences(cuda):
    torch = cuda
    from tdmd_claude_b200.fitting import eam_coeff_tensors, eam_table_meta
    pos, types, lo, hi, tgt = _snapshots(1, 31)
    _, eam = _tables(1)
    fm = _fm(pos, types, lo, hi, "fp64")
    fm.set_targets(tgt)
    meta = eam_table_meta(eam)
    F, rho, phi = eam_coeff_tensors(eam)
    _, gF, gr, gp = _eam_gpu(fm, torch, meta, F, rho, phi)
    rng = np.random.default_rng(3)
    for tens, g, name in ((F, gF, 0), (rho, gr, 1), (phi, gp, 2)):
        scale = np.abs(g[0]).max()
        nz = np.nonzero(np.abs(g[0]) > 1e-6 * scale)[0]
        for k in rng.choice(nz, size=3, replace=False):
            base = float(tens[0, k].item())
            h = 1e-6 * max(abs(base), 1e-3)
            tens[0, k] = base + h
            lp = _eam_gpu(fm, torch, meta, F, rho, phi)[0]
            tens[0, k] = base - h
            lm = _eam_gpu(fm, torch, meta, F, rho, phi)[0]
            tens[0, k] = base
            assert abs((lp - lm) / (2 * h) - g[0][k]) <= 1e-5 * scale, (name, k)


def test_autograd_wrappers_and_adam(cuda):
    torch = cuda
    from tdmd_claude_b200.fitting import adam_fit, eam_coeff_tensors, eam_loss, eam_table_meta
    from tdmd_claude_b200.fitting import morse_loss
    pos, types, lo, hi, _ = _snapshots(1, 41)
    fm = _fm(pos, types, lo, hi, "fp64")
    # Morse: targets from perturbed parameters; Adam moves toward them.
    true = np.array(MORSE[:3]) * np.array([1.05, 0.96, 1.03])
    fm.set_targets(fm.morse_forces(true))
    p = torch.tensor(MORSE[:3], dtype=torch.float64, device="cuda", requires_grad=True)
    loss = morse_loss(p, fm)
    loss.backward()
    _, g = _morse_gpu(fm, torch, MORSE[:3])
    assert np.allclose(p.grad.cpu().numpy(), g, rtol=1e-12, atol=0)
    p.grad = None
    losses, sec = adam_fit(lambda q: morse_loss(q, fm), [p], steps=200, lr=2e-3)
    assert losses[-1] < 0.1 * losses[0] and sec > 0
    # EAM: gradients through autograd equal the raw call; a few steps lower the loss.
    _, eam = _tables(1)
    meta = eam_table_meta(eam)
    F, rho, phi = (x.clone().requires_grad_(True) for x in eam_coeff_tensors(eam))
    fm.set_targets(np.random.default_rng(2).normal(0.0, 0.3, size=pos.shape))
    loss = eam_loss(F, rho, phi, fm, meta)
    loss.backward()
    _, gF, gr, gp = _eam_gpu(fm, torch, meta, F.detach(), rho.detach(), phi.detach())
    # FP64 atomics: the two gradients may differ in the last bits
    assert np.allclose(F.grad.cpu().numpy(), gF, rtol=1e-12, atol=1e-12 * np.abs(gF).max())
    losses, _ = adam_fit(lambda a, b, c: eam_loss(a, b, c, fm, meta), [F, rho, phi], steps=20,
                         lr=1e-4)
    assert losses[-1] < losses[0]


def test_eam_gradient_vs_oracle_many_atoms(cuda, oracle):
    """40,000 atoms (10 snapshots of 10^3 cells): the kernels run with 8
    lanes per atom here (the small cases above use 32)."""
    torch = cuda
    from tdmd_claude_b200.fitting import eam_coeff_tensors, eam_table_meta
    pos, types, lo, hi, tgt = _snapshots(1, 50, nsnap=10, ncell=10)
    t, eam = _tables(1)
    from tdmd_claude_b200 import Box
    from tdmd_claude_b200.fitting import ForceMatch
    fm = ForceMatch(pos, types, Box.make(lo, hi), t.cutoff, "fp64")
    fm.set_targets(tgt)
    F, rho, phi = eam_coeff_tensors(eam)
    loss, gF, gr, gp = _eam_gpu(fm, torch, eam_table_meta(eam), F, rho, phi)
    oe = oracle.OracleEam(t.ntypes, t.nrho, t.drho, t.nr, t.dr, t.cutoff, t.F, t.rho, t.rphi)
    lo_, oF, orho, ophi = oe.fm_loss_grad(pos, types, lo, hi, tgt)
    assert abs(loss - lo_) <= 1e-10 * lo_
    for got, ref in ((gF, oF), (gr, orho), (gp, ophi)):
        assert np.abs(got[0] - ref[0]).max() <= 1e-9 * np.abs(ref[0]).max()


def test_eam_fit_rejects_cutoff_past_tables(cuda):
    torch = cuda
    from tdmd_claude_b200 import TdmdError
    from tdmd_claude_b200.fitting import eam_coeff_tensors, eam_table_meta
    pos, types, lo, hi, tgt = _snapshots(1, 60)
    _, eam = _tables(1)
    fm = _fm(pos, types, lo, hi, "fp64")      # cutoff 5.0 = the tables' end: accepted
    fm.set_targets(tgt)
    F, rho, phi = eam_coeff_tensors(eam)
    _eam_gpu(fm, torch, eam_table_meta(eam), F, rho, phi)
    from tdmd_claude_b200 import Box
    from tdmd_claude_b200.fitting import ForceMatch
    far = ForceMatch(pos, types, Box.make(lo, hi), 5.2, "fp64")
    far.set_targets(tgt)
    with pytest.raises(TdmdError):
        _eam_gpu(far, torch, eam_table_meta(eam), F, rho, phi)


@pytest.mark.parametrize("ntypes", [1, 3])
def test_eam_gradient_run_to_run_spread(cuda, ntypes):
    """The EAM adjoint adds coefficient gradients with FP64 atomics (per
    block in shared memory, then once per block in global memory), so the
    order of those additions, and the last bits of the gradient, can change
    from call to call.  The loss and the Morse gradient are fixed-order.
    This states the spread: ten calls on the same inputs (64 snapshots of
    10^3 cells, the force-matching workload's size) differ by at most 1e-14
    of each spline's largest gradient entry; the loss is bit-identical."""
    torch = cuda
    from tdmd_claude_b200 import Box
    from tdmd_claude_b200.fitting import ForceMatch, eam_coeff_tensors, eam_table_meta
    pos, types, lo, hi, tgt = _snapshots(ntypes, 60 + ntypes, nsnap=16, ncell=10)
    t, eam = _tables(ntypes)
    fm = ForceMatch(pos, types, Box.make(lo, hi), t.cutoff, "fp64")
    fm.set_targets(tgt)
    F, rho, phi = eam_coeff_tensors(eam)
    meta = eam_table_meta(eam)
    runs = [_eam_gpu(fm, torch, meta, F, rho, phi) for _ in range(10)]
    l0, g0 = runs[0][0], runs[0][1:]
    worst = 0.0
    for loss, *g in runs[1:]:
        assert loss == l0
        for got, ref in zip(g, g0):
            for sp in range(ref.shape[0]):
                scale = np.abs(ref[sp]).max()
                if scale > 0:
                    worst = max(worst, float(np.abs(got[sp] - ref[sp]).max() / scale))
    assert worst <= 1e-14, worst
    print(f"EAM adjoint run-to-run spread (ntypes={ntypes}): {worst:.3e} of the largest entry")
