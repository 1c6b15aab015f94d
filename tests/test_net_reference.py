"""The numpy restatement of the warm-start network checks itself: its
back-propagated gradient against central finite differences in FP64, and its
site geometry against the fields' parity-split order (CPU only)."""
import numpy as np

import net_reference as NR


def _problem(L, seed):
    rng = np.random.default_rng(seed)
    V = L[0] * L[1] * L[2]
    feat = rng.standard_normal((V, 16))
    feat[:, 15] = 0.0
    t = rng.standard_normal((V, 4))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    w = rng.standard_normal(NR.NPARAM) * 0.2
    return w, feat, t


def test_neighbours_are_a_permutation_and_inverse():
    L = (4, 6, 4)
    nbr = NR.neighbours(L)
    V = 4 * 6 * 4
    for k in range(27):
        assert np.array_equal(np.sort(nbr[k]), np.arange(V))
        # offset 26-k undoes offset k
        assert np.array_equal(nbr[26 - k][nbr[k]], np.arange(V))
    assert np.array_equal(nbr[13], np.arange(V))


def test_coordinates_follow_parity_split_order():
    L = (4, 4, 6)
    x, y, z = NR.coords(L)
    nh = 48
    assert np.all(((x + y + z) & 1)[:nh] == 0) and np.all(((x + y + z) & 1)[nh:] == 1)
    assert np.array_equal(NR.flat_index(L, x, y, z), np.arange(96))


def test_gradient_matches_finite_differences():
    L = (4, 4, 4)
    w, feat, t = _problem(L, 3)
    _, loss, g = NR.forward_backward(w, feat, t, L, bf16_path=False)
    rng = np.random.default_rng(5)
    # sampled coordinates in every layer, weights and biases; output rows >= 4 have zero gradient
    idx = []
    for l in range(NR.LAYERS):
        base = l * NR.PL
        hi_co = NR.OUT if l == NR.LAYERS - 1 else 16
        for _ in range(6):
            k, co, ci = rng.integers(27), rng.integers(hi_co), rng.integers(16)
            idx.append(base + (k * 16 + co) * 16 + ci)
        idx.append(base + NR.WL + rng.integers(hi_co))
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (NR.loss_only(wp, feat, t, L) - NR.loss_only(wm, feat, t, L)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 3.14159])
    r = NR.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 4 * 2 ** -8    # tie to even (up)
    assert r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 3.14159) < 2 ** -7 * 3.2
