"""The hand-written adjoint of em2's step (maccpic_b200/adjoint.py).

* the plain-PyTorch step is em2's step: checked against the C oracle
  (pic/move.f90, pic/curnt.f90, pic/fields.f90) on a periodic state;
* the hand-written reverse of one step equals autograd's vector-Jacobian
  product of the PyTorch step, for random output adjoints;
* the checkpointed reverse sweep over T steps equals the FP64 autograd tape;
* d flux(T) / d theta agrees with central finite differences taken with
  common random numbers (h = 1e-3) to within 1 %.

All on the CPU at small sizes (FP64), plus the same gradient on the GPU.
"""
import numpy as np
import pytest
import torch

from maccpic_b200 import adjoint as A
from maccpic_b200 import loader

THETA = (0.1, 0.0, 0.5)          # psi0/(B0 d_i), B_g/B0, L/d_i of the nominal workload


def _cfg(**kw):
    base = dict(nx=32, ny=32, ppc=4, seed=3, isav=2)
    base.update(kw)
    return loader.HarrisConfig(**base)


def _guarded(a: torch.Tensor) -> np.ndarray:
    """Periodic (ny, nx) array -> em2's (0:ny+2, 0:nx+2) block with exact
    periodic images: index (ix, iy) holds periodic node (ix-1, iy-1)."""
    a = a.detach().cpu().numpy()
    ny, nx = a.shape
    iy = (np.arange(ny + 3) - 1) % ny
    ix = (np.arange(nx + 3) - 1) % nx
    return a[np.ix_(iy, ix)]


def _oracle_state(oracle, cfg, E, B, parts, cg_eps=1e-9):
    from oracle import NFIELD
    rp = cfg.run_params()
    op = oracle.Params(nx=cfg.nx, ny=cfg.ny, dx=rp.dx, dy=rp.dy, dt=rp.dt, qm=rp.qm, q=rp.q,
                       dn=rp.dn, am=rp.am, isav=cfg.isav, cg_eps=cg_eps)
    fld = np.zeros((NFIELD, cfg.ny + 3, cfg.nx + 3))
    for i, a in enumerate(list(E) + list(B)):
        fld[i] = _guarded(a)
    ps = []
    for (x, y, ux, uy, uz) in parts:
        g = torch.sqrt(1.0 + ux * ux + uy * uy + uz * uz)
        ps.append(torch.stack([x, y, ux / g, uy / g, uz / g, g]).detach().numpy().copy())
    return oracle.State(op, fld, ps)


def test_step_matches_oracle(oracle_lib):
    """Four steps (two of them with the isav field filter) of the PyTorch
    step against the oracle.  The PyTorch step solves the Poisson
    correction exactly (FFT); the oracle's CG is run to mean r^2 < 1e-26
    instead of em2's 1e-9 so that both are exact to rounding, and
    everything then agrees to rounding amplified over four steps."""
    cfg = _cfg()
    d = A.make_draws(cfg)
    k = A.step_const(cfg)
    E, B, P = A.initial_state_torch(cfg, THETA, d)
    st = _oracle_state(oracle_lib, cfg, E, B, P, cg_eps=1e-26)
    for it in range(1, 5):
        E, B, P = A.step(E, B, P, k, it)
        st.move()
        st.curnt()
        st.fields(it)
    for i, a in enumerate(list(E) + list(B)):
        ref = st.fld[i]
        got = _guarded(a)
        scale = max(np.abs(ref).max(), 1e-3)
        assert np.abs(got - ref).max() / scale < 1e-9, i
    for s, (x, y, ux, uy, uz) in enumerate(P):
        o = st.parts[s]
        dxp = np.abs(x.numpy() - o[0])
        dxp = np.minimum(dxp, cfg.nx - dxp)        # a wrap may land on either side
        dyp = np.abs(y.numpy() - o[1])
        dyp = np.minimum(dyp, cfg.ny - dyp)
        assert dxp.max() < 1e-11 and dyp.max() < 1e-11
        g = torch.sqrt(1.0 + ux * ux + uy * uy + uz * uz).numpy()
        for c, u in enumerate((ux, uy, uz)):
            assert np.abs(u.numpy() / g - o[2 + c]).max() < 1e-11


def _rand_like_state(E, B, P, gen):
    r = lambda t: torch.randn(t.shape, generator=gen, dtype=t.dtype)
    return tuple(r(e) for e in E), tuple(r(b) for b in B), [tuple(r(t) for t in p) for p in P]


@pytest.mark.parametrize("it", [1, 2])       # it = 2: with the isav E/B filter
def test_step_T_is_the_vjp(it):
    cfg = _cfg()
    d = A.make_draws(cfg)
    k = A.step_const(cfg)
    E, B, P = A.initial_state_torch(cfg, THETA, d)
    with torch.no_grad():                       # a state with particles off the lattice
        E, B, P = A.step(E, B, P, k, 1)
    gen = torch.Generator().manual_seed(5)
    lE2, lB2, lP2 = _rand_like_state(E, B, P, gen)
    leaves = [t.detach().clone().requires_grad_(True) for t in A._flatten(E, B, P)]
    Ei, Bi, Pi = A._unflatten(leaves, 2)
    out = A._flatten(*A.step(Ei, Bi, Pi, k, it))
    vjp = torch.autograd.grad(out, leaves, grad_outputs=A._flatten(lE2, lB2, lP2),
                              allow_unused=True)
    with torch.no_grad():
        mine = A._flatten(*A.step_T(E, B, P, lE2, lB2, lP2, k, it))
    for a, b in zip(mine, vjp):
        b = torch.zeros_like(a) if b is None else b
        assert float((a - b).abs().max()) <= 1e-12 * max(float(b.abs().max()), 1.0)


def test_autograd_function_backward():
    """Em2Step's backward (the hand-written reverse) through autograd."""
    cfg = _cfg(nx=16, ny=16, ppc=2)
    d = A.make_draws(cfg)
    k = A.step_const(cfg)
    E, B, P = A.initial_state_torch(cfg, THETA, d)
    leaves = [t.detach().clone().requires_grad_(True) for t in A._flatten(E, B, P)]
    out = A.Em2Step.apply(k, 1, 2, *leaves)
    _, B2, _ = A._unflatten(list(out), 2)
    F = A.flux(B2, k)
    g = torch.autograd.grad(F, leaves, allow_unused=True)
    Fr, ref = A._reference_tape(E, B, P, k, 1)
    assert float(F.detach()) == pytest.approx(float(Fr), rel=1e-14)
    for a, b in zip(g, A._flatten(*ref)):
        a = torch.zeros_like(b) if a is None else a
        assert float((a - b).abs().max()) <= 1e-12 * max(float(b.abs().max()), 1.0)


def test_checkpointed_sweep_matches_autograd_tape():
    cfg = _cfg()
    d = A.make_draws(cfg)
    k = A.step_const(cfg)
    E, B, P = A.initial_state_torch(cfg, THETA, d)
    steps = 9
    F, lE, lB, lP = A.flux_and_gradient(E, B, P, k, steps, checkpoint=4)
    Fr, (gE, gB, gP) = A._reference_tape(E, B, P, k, steps)
    assert float(F) == float(Fr)
    for a, b in zip(A._flatten(lE, lB, lP), A._flatten(gE, gB, gP)):
        assert float((a - b).abs().max()) <= 1e-11 * max(float(b.abs().max()), 1e-300)


def test_theta_gradient_matches_central_differences():
    cfg = _cfg()
    d = A.make_draws(cfg)
    steps, h = 12, 1e-3
    F, g = A.theta_gradient(cfg, THETA, steps, checkpoint=5, draws=d)
    assert F == pytest.approx(A.flux_of_theta(cfg, THETA, steps, d), rel=1e-13)
    for i in range(3):
        tp, tm = list(THETA), list(THETA)
        tp[i] += h
        tm[i] -= h
        fd = (A.flux_of_theta(cfg, tp, steps, d) - A.flux_of_theta(cfg, tm, steps, d)) / (2 * h)
        # psi0 and L dominate; the guide-field derivative is tiny at B_g = 0
        assert abs(g[i] - fd) <= 0.01 * abs(fd) + 1e-9, (i, g[i], fd)


@pytest.mark.gpu
def test_theta_gradient_on_gpu_matches_cpu(gpu):
    cfg = _cfg()
    steps = 6
    Fc, gc = A.theta_gradient(cfg, THETA, steps, checkpoint=3, draws=A.make_draws(cfg))
    Fg, gg = A.theta_gradient(cfg, THETA, steps, checkpoint=3,
                              draws=A.make_draws(cfg, device="cuda"), device="cuda")
    assert Fg == pytest.approx(Fc, rel=1e-10)
    np.testing.assert_allclose(gg, gc, rtol=1e-7, atol=1e-12)
