"""The CUDA adjoint (em2g_adj_*, maccpic_b200/adjoint.py CudaAdjoint).

* the FP64 CUDA step with the exact Poisson solve is the PyTorch step of
  maccpic_b200/adjoint.py (to round-off);
* one reverse step equals the hand-written PyTorch reverse step_T, itself
  checked against autograd (tests/test_adjoint.py);
* the whole sweep (rebuilt states, checkpoints, regrouping) gives the
  PyTorch adjoint's d flux / d theta;
* d flux / d theta agrees with central differences of the CUDA forward
  (common random numbers, h = 1e-3) to within 1 %, and over a longer
  horizon with h = 1e-6 to 1e-3.
"""
import numpy as np
import pytest
import torch

from maccpic_b200 import adjoint as A
from maccpic_b200 import loader

pytestmark = pytest.mark.gpu

THETA = (0.1, 0.0, 0.5)


def _cfg(**kw):
    base = dict(nx=32, ny=32, ppc=4, seed=3, isav=2)
    base.update(kw)
    return loader.HarrisConfig(**base)


def _state(cfg):
    d = A.make_draws(cfg, device="cuda")
    k = A.step_const(cfg)
    E, B, P = A.initial_state_torch(cfg, THETA, d)
    return k, E, B, P


def rel(a, b):
    return float((a - b).abs().max()) / max(float(b.abs().max()), 1e-300)


def test_spectral_step_matches_torch_step(gpu):
    cfg = _cfg()
    k, E, B, P = _state(cfg)
    with A.CudaAdjoint(k, E, B, P, 1, 1, cfg.isav) as adj:
        for it in range(1, 5):
            E, B, P = A.step(E, B, P, k, it)
            adj.g.step(1)
        fld = adj.g.get_fields()
        for c, a in enumerate(list(E) + list(B)):
            got = torch.from_numpy(fld[c, 1:k.ny + 1, 1:k.nx + 1]).to(a.device)
            assert rel(got, a) < 1e-10, c
        for s, (x, y, ux, uy, uz) in enumerate(P):
            q = torch.from_numpy(adj.g.get_particles(s)).to(x.device)
            dx = (q[0] - x).abs()
            assert float(torch.minimum(dx, k.nx - dx).max()) < 1e-11
            dy = (q[1] - y).abs()
            assert float(torch.minimum(dy, k.ny - dy).max()) < 1e-11
            for c, u in enumerate((ux, uy, uz)):
                assert float((q[2 + c] * q[5] - u).abs().max()) < 1e-11


@pytest.mark.parametrize("isav", [1, 2])   # it = 1: with and without the E/B filter
def test_one_reverse_step_matches_step_T(gpu, isav):
    cfg = _cfg(isav=isav)
    k, E, B, P = _state(cfg)
    with torch.no_grad():
        E, B, P = A.step(E, B, P, k, 1)      # a state with particles off the lattice
    gen = torch.Generator(device="cuda").manual_seed(7)
    lE2 = tuple(torch.randn(e.shape, generator=gen, dtype=e.dtype, device=e.device) for e in E)
    lB2 = tuple(torch.randn(b.shape, generator=gen, dtype=b.dtype, device=b.device) for b in B)
    zero = [tuple(torch.zeros_like(t) for t in p) for p in P]
    import ctypes as C
    from maccpic_b200._lib import check
    with A.CudaAdjoint(k, E, B, P, 1, 1, isav, it0=1) as adj:
        adj.forward(1)
        # the state as the CUDA adjoint saw it (u = (u/gamma) gamma)
        P_cuda = []
        for s in range(len(P)):
            x = torch.empty((5, adj.n[s]), dtype=torch.float64, device="cuda")
            check(adj._L.em2g_adj_get_initial_particles_device(
                adj._h, s, *[C.c_void_p(x[c].data_ptr()) for c in range(5)]))
            P_cuda.append(tuple(x[c] for c in range(5)))
        lE, lB, lP = adj.backward(lE2, lB2)
    with torch.no_grad():
        rE, rB, rP = A.step_T(E, B, P_cuda, lE2, lB2, zero, k, 2)
    for a, b in zip(list(lE) + list(lB), list(rE) + list(rB)):
        assert rel(a, b) < 1e-9
    for s in range(len(P)):
        for a, b in zip(lP[s], rP[s]):
            assert rel(a, b) < 1e-8


def test_sweep_matches_torch_gradient(gpu):
    cfg = _cfg()
    d = A.make_draws(cfg, device="cuda")
    steps = 12
    F_t, g_t = A.theta_gradient(cfg, THETA, steps, checkpoint=5, draws=d, device="cuda")
    F_c, g_c = A.theta_gradient_cuda(cfg, THETA, steps, checkpoint=5, draws=d)
    assert F_c == pytest.approx(F_t, rel=1e-10)
    np.testing.assert_allclose(g_c, g_t, rtol=1e-7, atol=1e-12)


def test_cuda_gradient_matches_central_differences(gpu):
    cfg = _cfg(nx=64, ny=64, ppc=8, seed=11, isav=20)
    d = A.make_draws(cfg, device="cuda")
    steps, h = 30, 1e-3
    F, g = A.theta_gradient_cuda(cfg, THETA, steps, checkpoint=10, draws=d)
    assert F == pytest.approx(A.flux_of_theta_cuda(cfg, THETA, steps, d), rel=1e-12)
    for i in range(3):
        tp, tm = list(THETA), list(THETA)
        tp[i] += h
        tm[i] -= h
        fd = (A.flux_of_theta_cuda(cfg, tp, steps, d)
              - A.flux_of_theta_cuda(cfg, tm, steps, d)) / (2 * h)
        assert abs(g[i] - fd) <= 0.01 * abs(fd) + 1e-9, (i, g[i], fd)


def test_long_horizon_gradient_matches_small_step_differences(gpu):
    """Over a horizon where the flux is no longer linear in theta across
    +-1e-3, the adjoint is still the derivative: central differences with
    h = 1e-6 (common random numbers, FP64 round-off ~1e-16 flux / h) agree
    with it to 1e-3 relative, through a workspace that recomputes segments."""
    cfg = _cfg(nx=64, ny=64, ppc=8, seed=11, isav=20)
    d = A.make_draws(cfg, device="cuda")
    k = A.step_const(cfg)
    steps = 300
    with A.CudaAdjoint(k, *A.initial_state_torch(cfg, THETA, d), steps, 50, cfg.isav,
                       field_slots=50) as ws:
        r = A.fd_check_cuda(cfg, THETA, steps, h=1e-6, checkpoint=50, draws=d, workspace=ws)
    assert max(r["rel_error"]) < 1e-3, r


def test_reused_workspace_gives_the_same_gradient(gpu):
    cfg = _cfg()
    d = A.make_draws(cfg, device="cuda")
    k = A.step_const(cfg)
    F0, g0 = A.theta_gradient_cuda(cfg, THETA, 8, checkpoint=4, draws=d)
    with A.CudaAdjoint(k, *A.initial_state_torch(cfg, THETA, d), 10, 4, cfg.isav) as ws:
        for theta in (THETA, (0.12, 0.05, 0.55), THETA):
            F, g = A.theta_gradient_cuda(cfg, theta, 8, checkpoint=4, draws=d, workspace=ws)
        assert F == pytest.approx(F0, rel=1e-13)
        np.testing.assert_allclose(g, g0, rtol=1e-9, atol=1e-13)
        with pytest.raises(ValueError):
            A.theta_gradient_cuda(cfg, THETA, 12, checkpoint=4, draws=d, workspace=ws)


def test_recomputed_segments_match_kept_fields(gpu):
    """Checkpoints every K steps with E and B of the last n steps kept and
    the steps before them recomputed from their checkpoints give the
    gradient that keeping E and B of every step gives, for n = K (the least
    memory), an n that splits a segment, and every step; each leaves the
    context at the final state the forward sweep reached."""
    cfg = _cfg()
    d = A.make_draws(cfg, device="cuda")
    k = A.step_const(cfg)
    steps, K = 12, 5                      # segments of 5, 5 and 2 steps
    E0, B0, P0 = A.initial_state_torch(cfg, THETA, d)
    grads = []
    # 12 slots: nothing recomputed; 8: steps 0-3 (part of the first segment);
    # 5: steps 0-6 (a whole segment and part of the next)
    for slots in (steps, 8, K):
        with A.CudaAdjoint(k, E0, B0, P0, steps, K, cfg.isav, field_slots=slots) as adj:
            assert adj.field_slots() == slots
            adj.forward(steps)
            Ef, Bf = adj.final_EB()
            seed = [torch.ones_like(b) * 1e-3 for b in Bf]
            lE, lB, lP = adj.backward([torch.zeros_like(e) for e in Ef], seed)
            Ef2, Bf2 = adj.final_EB()
            for a, b in zip(Ef + Bf, Ef2 + Bf2):
                assert torch.equal(a, b)
            assert adj.g.it == steps
            grads.append([t.clone() for t in list(lE) + list(lB) + [x for p in lP for x in p]])
    for other in grads[1:]:
        for a, b in zip(grads[0], other):
            assert rel(a, b) < 1e-9


def test_field_slots_bounds_and_default(gpu):
    """Slots are bounded by the checkpoint interval and max_steps; the
    default holds every step when they fit, and keep_all_fields is
    max_steps."""
    from maccpic_b200._lib import Em2gError
    cfg = _cfg()
    d = A.make_draws(cfg, device="cuda")
    k = A.step_const(cfg)
    E0, B0, P0 = A.initial_state_torch(cfg, THETA, d)
    with A.CudaAdjoint(k, E0, B0, P0, 12, 5, cfg.isav) as adj:
        assert adj.field_slots() == 12          # a few MB: every step fits
        for bad in (4, 13):
            with pytest.raises(Em2gError):
                adj.set_field_slots(bad)
        adj.set_field_slots(5)
        assert adj.field_slots() == 5
        assert adj.slots_that_fit(0.0) == 5
    with A.CudaAdjoint(k, E0, B0, P0, 12, 5, cfg.isav, keep_all_fields=True) as adj:
        assert adj.field_slots() == 12


def test_autograd_function_reaches_theta(gpu):
    """flux.backward() through CudaRun reaches the initial-state parameters,
    and a second backward through a fresh graph gives the same gradient."""
    cfg = _cfg()
    d = A.make_draws(cfg, device="cuda")
    k = A.step_const(cfg)
    with A.CudaAdjoint(k, *A.initial_state_torch(cfg, THETA, d), 8, 4, cfg.isav) as adj:
        gs = []
        for _ in range(2):
            th = torch.tensor(THETA, dtype=torch.float64, device="cuda", requires_grad=True)
            E0, B0, P0 = A.initial_state_torch(cfg, (th[0], th[1], th[2]), d)
            out = A.CudaRun.apply(adj, 8, *A.flatten_state(E0, B0, P0))
            A.flux(out[3:], k).backward()
            assert th.grad is not None and torch.isfinite(th.grad).all()
            gs.append(th.grad.clone())
    assert torch.allclose(gs[0], gs[1], rtol=1e-12, atol=0)
    assert gs[0].abs().max() > 0
