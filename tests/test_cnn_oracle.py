"""The CPU oracle of the learned proposal network checks itself: its
backward pass is the derivative of its loss (central finite differences
without BF16 rounding), its BF16 rounding is round-to-nearest-even, and a
label owns its 4x4 cell with the lowest index winning."""
import numpy as np

from oracle import cnn_oracle as co


def test_gradient_is_derivative_of_loss():
    rng = np.random.default_rng(0)
    n = co.num_params()
    p = rng.normal(0, 0.2, n)
    x = rng.normal(0, 1, (2, 5, 6, 16))
    tgt = np.zeros((2, 5, 6, 3))
    tgt[0, 2, 3] = (1, 0.3, -0.7)
    tgt[1, 1, 1] = (1, -1.0, 0.5)
    (ls, lo), g = co.loss_grad(p, x, tgt, 8.0, 1.0, exact=True)
    assert ls > 0 and lo > 0
    errs = []
    for i in rng.choice(n, 40, replace=False):
        e = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        (a, b), _ = co.loss_grad(pp, x, tgt, 8.0, 1.0, exact=True)
        (c, d), _ = co.loss_grad(pm, x, tgt, 8.0, 1.0, exact=True)
        fd = ((a + b) - (c + d)) / (2 * e)
        errs.append(abs(fd - g[i]) / max(1e-6, abs(fd) + abs(g[i])))
    assert max(errs) < 5e-3


def test_bf16_rounding_ties_to_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0], np.float32)
    r = co.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie, even mantissa stays
    assert r[2] == np.float32(1.0 + 4 * 2 ** -8)  # tie, odd mantissa rounds up
    assert r[3] == 1.0
    assert r[4] == -2.5 and r[5] == 0.0


def test_targets_lowest_label_owns_cell():
    t = co.targets([0, 0, 1], [5.2, 6.9, 1.0], [9.0, 8.1, 2.0], 2, 4, 4)
    assert t[0, 1, 2, 0] == 1.0
    assert np.isclose(t[0, 1, 2, 1], 5.2 - 5.5) and np.isclose(t[0, 1, 2, 2], 9.0 - 9.5)
    assert t[1, 0, 0, 0] == 1.0 and t.sum(axis=(1, 2, 3))[0] != 0


def test_cells_layout_and_padding():
    f = np.arange(2 * 6 * 7, dtype=np.uint16).reshape(2, 6, 7)
    c = co.cells(f, 0.0, 1.0)
    assert c.shape == (2, 2, 2, 16)
    assert c[0, 0, 0, 4 * 1 + 2] == f[0, 1, 2]
    assert c[1, 1, 1, 4 * 1 + 2] == f[1, 5, 6]
    assert c[1, 1, 1, 4 * 2 + 0] == 0.0   # row 6 is outside the frame: the mean
