"""CPU checks of the denoiser oracle: its analytic gradient against central
finite differences of the exact network, bf16 rounding, octahedral encoding
and the neighbourhood rows on a hand-made image."""
import numpy as np

from oracle import denoise as D


def small_problem(seed=0, m=24):
    rng = np.random.default_rng(seed)
    p = D.init_params(seed).astype(np.float64)
    q = D.unpack(p, np.float64)
    q["b1"][:] = rng.normal(0, 0.1, 64)
    q["b2"][:] = rng.normal(0, 0.1, 64)
    q["b3"][:] = rng.normal(0, 0.1, 4)
    x = np.zeros((m, 256))
    x[:, :250] = rng.normal(0, 1, (m, 250))
    t = rng.normal(0, 0.3, (m, 4))
    return p, x, t


def test_gradient_matches_finite_differences():
    p, x, t = small_problem()
    g, loss = D.backward(p, x, t, bf=False)
    assert abs(loss - D.loss_of(p, x, t)) < 1e-12
    rng = np.random.default_rng(1)
    # a sample of parameters from every block, W1's pad columns excluded
    picks = []
    for name, (off, shape) in D.LAYOUT.items():
        n = int(np.prod(shape))
        cand = np.arange(off, off + n)
        if name == "w1":
            cand = cand[(cand - off) % 256 < 250]
        picks += list(rng.choice(cand, min(12, len(cand)), replace=False))
    h = 1e-6
    for i in picks:
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        fd = (D.loss_of(a, x, t) - D.loss_of(b, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    assert np.all(g[:16384].reshape(64, 256)[:, 250:] == 0)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0, 1.0 + 2 ** -8 + 2 ** -20],
                 np.float32)
    got = D.bf16(v)
    want = np.array([1.0, 1.0, 1.0 + 4 * 2 ** -8, 1.0, -2.5, 0.0, 1.0 + 2 ** -7], np.float32)
    assert np.array_equal(got, want)


def test_octahedral_encoding():
    v = np.array([[0, 0, 1], [0, 0, -1], [1, 0, 0], [0, 0, 0], [np.nan, 0, 0], [1, 1, -2]], np.float32)
    ox, oy = D.oct_encode(v)
    assert np.allclose(ox, [0, 1, 1, 0, 0, 0.75]) and np.allclose(oy, [0, 1, 0, 0, 0, 0.75])


def test_rows_neighbourhood_and_padding():
    w, h = 6, 5
    n = w * h
    idx = np.arange(n, dtype=np.uint32)
    tidx = np.zeros(n, np.uint32)
    tidx[7] = D.MISS  # pixel (1, 1) has no mapping hit
    ao = np.linspace(0, 1, n, dtype=np.float32)
    bn = np.tile(np.array([0, 0, 1], np.float32), n)
    pos = np.stack([np.arange(n) % w, np.arange(n) // w, np.zeros(n)], 1).astype(np.float32).reshape(-1)
    nrm = np.tile(np.array([0, 0, 1], np.float32), n)
    coords = np.zeros((n, 4), np.float32)
    coords[:, 0] = 0.25
    f = D.features(w, h, idx, tidx, coords, ao, bn, pos, nrm, 0.5)
    x = D.rows(f, w, h, np.array([0, 14, 0xFFFFFFFF], np.uint32))
    r = x[:, :250].reshape(3, 25, 10)
    assert np.all(x[:, 250:] == 0) and np.all(r[2] == 0)
    # corner pixel: only the 3 x 3 lower-right part of the window is inside, (1,1) has no hit
    inside = [(dy, dx) for dy in range(3) for dx in range(3) if (dy, dx) != (1, 1)]
    for j in range(25):
        dx, dy = j % 5 - 2, j // 5 - 2
        exp = (dy, dx) in inside
        assert (r[0, j, 9] == 1) == exp
    # centre (2, 2) of pixel 14: texel spacing 1 / 0.5 = 2 in position / R units, so neighbour (+1, +2) sits
    # at (1, 2) spacings
    assert f[2, 14, 2] == 2.0 and f[2, 8, 2] == 2.0  # pixel 8 = (2, 1) averages 3 covered neighbours
    j = (2 + 2) * 5 + (1 + 2)
    assert np.allclose(r[1, j, 3:6], [1.0, 2.0, 0.0])
    assert r[1, 12, 8] == D.bf16(np.float32(0.25) / np.float32(0.5))
