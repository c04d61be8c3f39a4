"""The differentiation form: the hand-written adjoint of the RHS against
torch autograd through the FP64 torch restatement (oracle/tdgl_torch_ref.py),
which is itself pinned to the reference's golden RHS vectors.

Tolerances: RHS restatement 1e-14 relative (summation order); adjoint
gradients 1e-11 relative to the largest entry (FP64 atomics reorder sums).
"""

import numpy as np
import pytest
import torch

from conftest import device_from_fixture, golden, golden_names
from oracle import tdgl_oracle as orc
from oracle import tdgl_torch_ref as tr

CASES = golden_names("case_")


@pytest.mark.parametrize("name", CASES)
def test_torch_restatement_matches_golden_rhs(name):
    d = golden(name)
    dev = device_from_fixture(d)
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    B = [float(v) for v in d["B"]]
    for key in ("X_seeded", "X_random"):
        if key not in d:
            continue
        X = d[key]
        sc = None if g.sc_int is None else torch.tensor(g.sc_int)
        f = tr.eval_f(g, torch.tensor(tr.to_real(X, g)), sc, *B).numpy()
        ref = d["F_" + key[2:]] if ("F_" + key[2:]) in d else orc.eval_f(X, g, *B)
        err = np.max(np.abs(tr.from_real(f, g) - ref)) / max(np.max(np.abs(ref)), 1e-300)
        assert err < 1e-14, (name, key, err)


def _perm_dev_to_ref(grid, a_dev_order):
    """Per-node array in device order -> reference order (through unpack)."""
    v = grid.empty_state()
    v[:grid.n] = a_dev_order
    return grid.unpack(v).real[:grid.n]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_vjp_kernel_matches_autograd(name):
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200.engine import grid_for
    d = golden(name)
    dev = device_from_fixture(d)
    p = dev.params
    g = orc.make_grid(p, dev.idx, dev.material)
    B = [float(v) for v in d["B"]]
    if abs(B[0]) + abs(B[1]) + abs(B[2]) == 0.0:
        B = [0.11, -0.07, 0.23]                      # exercise every face offset
    grid = grid_for(p, dev.idx, dev.material, "fp64", 8)
    rng = np.random.default_rng(7)
    X = d["X_seeded"]
    nc = 5 if g.is_3d else 4
    v_real = rng.standard_normal(nc * g.n)
    # kernel
    x_dev = grid.pack(X)
    v_dev = grid.pack(tr.from_real(v_real, g))
    gx, gsc, gk2, gpar = grid.vjp(x_dev, v_dev, B)
    gx_real = tr.to_real(grid.unpack(gx).cpu().numpy(), g)
    # autograd
    xt = torch.tensor(tr.to_real(X, g), requires_grad=True)
    bt = [torch.tensor(b, dtype=torch.float64, requires_grad=True) for b in B]
    kt = None if g.kappa_int is not None else torch.tensor(g.kappa, dtype=torch.float64, requires_grad=True)
    sct = None if g.sc_int is None else torch.tensor(g.sc_int, requires_grad=True)
    f = tr.eval_f(g, xt, sct, *bt, kappa=kt)
    (f * torch.tensor(v_real)).sum().backward()
    ref = xt.grad.numpy()
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(gx_real - ref)) < 1e-11 * scale, np.max(np.abs(gx_real - ref)) / scale
    gp = gpar.cpu().numpy()
    for a in range(3):
        r = 0.0 if bt[a].grad is None else bt[a].grad.item()      # Bx, By do not enter a 2-D film
        assert abs(gp[a] - r) < 1e-10 * max(abs(r), 1.0), (a, gp[a], r)
    if kt is not None:
        assert abs(gp[3] - kt.grad.item()) < 1e-10 * max(abs(kt.grad.item()), 1.0)
    if sct is not None:
        gs = _perm_dev_to_ref(grid, gsc).cpu().numpy()
        r = sct.grad.numpy()
        assert np.max(np.abs(gs - r)) < 1e-11 * max(np.max(np.abs(r)), 1.0)


@pytest.mark.gpu
def test_autograd_function_matches_torch_reference():
    import nanowire_tdgl_b200 as tb
    d = golden("case_3d_hole")
    dev = device_from_fixture(d)
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    rng = np.random.default_rng(3)
    x = torch.tensor(tr.to_real(d["X_seeded"], g))
    w = torch.tensor(rng.standard_normal(x.numel()))
    B = [torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in (0.05, -0.1, 0.3)]
    xa = x.clone().requires_grad_(True)
    fa = tb.rhs(xa.cuda(), dev.params, dev.idx, dev.material, B)
    (fa.cpu() * w).sum().backward()
    xb = x.clone().requires_grad_(True)
    Bb = [b.detach().clone().requires_grad_(True) for b in B]
    sc = None if g.sc_int is None else torch.tensor(g.sc_int)
    fb = tr.eval_f(g, xb, sc, *Bb)
    assert torch.allclose(fa.cpu(), fb, rtol=0, atol=1e-12 * float(fb.abs().max()))
    (fb * w).sum().backward()
    assert torch.allclose(xa.grad, xb.grad, rtol=0, atol=1e-11 * float(xb.grad.abs().max()))
    for a, b in zip(B, Bb):
        assert abs(float(a.grad) - float(b.grad)) <= 1e-10 * max(abs(float(b.grad)), 1.0)
