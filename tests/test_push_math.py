"""The FP32 push's per-particle arithmetic restated in numpy float32 (CPU),
against em2's forms in FP64.

The push (maccpic_b200/csrc/push_f32_body.cuh, weights2 and split_cell)
takes em2's quadratic-spline weights (pic/move.f90:76-84: 3/4-d^2 at the
nearest node, (1/2-+d)^2/2 at its neighbours, d the offset from that node)
in another order of operations: the middle weight s = 3/4 - d^2,
t = (1 - s)/2, and the ends t -+ d/2, since the three sum to 1 and the ends differ by d.  Each packed
FP32 operation rounds as its scalar counterpart, so float32 numpy with the
same order is the kernel's arithmetic.  Checked here: the restated weights
equal em2's to FP32 rounding over the cell and sum to 1 to FP32 rounding,
and the cell split by floor gives a step of -1, 0 or 1 and an offset in
[0, 1] (1 only by rounding, which the grouping rules absorb) over the whole
(-1, 2) range the grouping allows.
"""
import numpy as np

F = np.float32


def weights_kernel(f):
    """weights2's half-node and integer-node weights of offsets f (float32)."""
    f = f.astype(F)
    d = f + F(-0.5)
    # each fma2 rounds once: emulated by the float64 result rounded to float32
    hs = (np.float64(0.75) - d.astype(np.float64) ** 2).astype(F)
    ht = (np.float64(0.5) - 0.5 * hs.astype(np.float64)).astype(F)
    hm = (ht.astype(np.float64) - 0.5 * d.astype(np.float64)).astype(F)
    hp = (ht.astype(np.float64) + 0.5 * d.astype(np.float64)).astype(F)
    u = (f >= F(0.5))
    h = f + np.where(u, F(-1.0), F(0.0))
    ns = (np.float64(0.75) - h.astype(np.float64) ** 2).astype(F)
    nt = (np.float64(0.5) - 0.5 * ns.astype(np.float64)).astype(F)
    nm = (nt.astype(np.float64) - 0.5 * h.astype(np.float64)).astype(F)
    np_ = (nt.astype(np.float64) + 0.5 * h.astype(np.float64)).astype(F)
    return (hm, hs, hp), (nm, ns, np_), u


def weights_em2(f):
    """em2's forms in FP64: cell-centred nodes about f - 1/2, integer nodes
    about the nearest node (f - u)."""
    f = f.astype(np.float64)
    d = f - 0.5
    half = ((0.5 - d) ** 2 / 2, 0.75 - d * d, (0.5 + d) ** 2 / 2)
    h = f - (f >= 0.5)
    node = ((0.5 - h) ** 2 / 2, 0.75 - h * h, (0.5 + h) ** 2 / 2)
    return half, node


def test_restated_weights_equal_em2s_to_fp32_rounding():
    rng = np.random.default_rng(7)
    f = np.concatenate([rng.random(200000), np.array([0.0, 0.5, 0.25, 0.75]),
                        np.nextafter(F(1.0), F(0.0), dtype=F)[None],
                        np.nextafter(F(0.5), F(0.0), dtype=F)[None]]).astype(F)
    (hm, hs, hp), (nm, ns, np_), _ = weights_kernel(f)
    half, node = weights_em2(f)
    for got, want in zip((hm, hs, hp, nm, ns, np_), half + node):
        assert np.abs(got.astype(np.float64) - want).max() < 1.2e-7
        assert got.min() >= 0.0
    # the three of each staggering sum to 1 (to FP32 rounding, the packed
    # sums being exact for these values)
    for a, b, c in ((hm, hs, hp), (nm, ns, np_)):
        s = a.astype(np.float64) + b + c
        assert np.abs(s - 1.0).max() < 1.2e-7


def test_cell_split_by_floor_covers_the_grouping_range():
    rng = np.random.default_rng(8)
    x = (rng.random(200000) * 3.0 - 1.0).astype(F)  # offsets in (-1, 2)
    x = np.concatenate([x, np.array([-0.9999999, 0.0, 0.9999999, 1.0, 1.9999999], dtype=F)])
    fl = np.floor(x)
    rest = (x - fl).astype(F)
    assert set(np.unique(fl)) <= {F(-1.0), F(0.0), F(1.0)}
    assert rest.min() >= 0.0 and rest.max() <= 1.0
    # the float cell step is exact, so the write-back's offset (rest + step)
    # lands within one rounding of the offset it came from
    assert np.abs((rest + fl).astype(np.float64) - x.astype(np.float64)).max() < 1.2e-7
