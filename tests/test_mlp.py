"""The learned troubled-cell indicator: a numpy restatement of the network,
its BF16 roundings and its gradient, checked against the library's
tensor-core training and inference kernels; the indicator's inputs against a
numpy restatement; and the learned limiter mode against the reference's
detectors at the thresholds where it must reproduce them exactly.

The network (no counterpart in the reference): p = sigmoid(w3 . gelu(gelu(X W1
+ b1) W2 + b2) + b3), 90-64-64-1. The products run as BF16 x BF16 with FP32
accumulation; X, W1, W2, w3, the first hidden layer and the back-propagated
dZ2, dZ1 are rounded to BF16, everything else is FP32. Loss: weighted binary
cross-entropy, mean over the batch, positives weighted by pos_weight."""
import numpy as np
import pytest
from scipy.special import erf

NIN, NH = 90, 64
OFF_W1 = 0
OFF_B1 = NIN * NH
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1


def bf16(x):
    """Round float32 to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p)
    return (p[OFF_W1:OFF_B1].reshape(NIN, NH), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NH, NH),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def gelu(x):
    return 0.5 * x * (1 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


def forward_backward(p, X, y, pos_weight=1.0, rounded=True):
    """(loss, gradient, probabilities). rounded=True restates the kernels'
    BF16 roundings in FP32; rounded=False is the plain FP64 model."""
    if rounded:
        dt, rnd = np.float32, bf16
    else:
        dt, rnd = np.float64, (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, w3, b3 = unpack(np.asarray(p, dt))
    X = rnd(np.asarray(X, dt))
    W1r, W2r, w3r = rnd(W1), rnd(W2), rnd(w3)
    n = len(y)
    wts = np.where(y > 0.5, pos_weight, 1.0).astype(dt)
    z1 = (X @ W1r + b1).astype(dt)
    h1 = rnd(gelu(z1).astype(dt))
    z2 = (h1 @ W2r + b2).astype(dt)
    h2 = gelu(z2).astype(dt)
    z3 = (h2 @ w3r + b3).astype(dt)
    pr = 1 / (1 + np.exp(-z3))
    sp = np.maximum(z3, 0) + np.log1p(np.exp(-np.abs(z3)))
    loss = float(np.sum(wts * (y * (sp - z3) + (1 - y) * sp)) / n)
    g3 = (wts * (pr - y) / n).astype(dt)
    dz2 = ((g3[:, None] * w3r[None, :]) * gelu_d(z2)).astype(dt)
    g = np.zeros(NPARAM, dt)
    g[OFF_B3] = g3.sum()
    g[OFF_W3:OFF_B3] = (g3[:, None] * h2).sum(0)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz2r = rnd(dz2)
    g[OFF_W2:OFF_B2] = (h1.T @ dz2r).ravel()
    dz1 = ((dz2r @ W2r.T) * gelu_d(z1)).astype(dt)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (X.T @ rnd(dz1)).ravel()
    return loss, g, pr


def glorot(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM)
    a1, a2, a3 = np.sqrt(6 / (NIN + NH)), np.sqrt(6 / (2 * NH)), np.sqrt(6 / (NH + 1))
    p[OFF_W1:OFF_B1] = rng.uniform(-a1, a1, NIN * NH)
    p[OFF_W2:OFF_B2] = rng.uniform(-a2, a2, NH * NH)
    p[OFF_W3:OFF_B3] = rng.uniform(-a3, a3, NH)
    p[OFF_B1:OFF_W2] = rng.normal(0, 0.1, NH)
    p[OFF_B2:OFF_W3] = rng.normal(0, 0.1, NH)
    p[OFF_B3] = 0.2
    return p


def batch(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, NIN)).astype(np.float32)
    y = (X[:, :8].sum(1) + 0.5 * rng.normal(size=n) > 1.0).astype(np.float32)
    return X, y


# ------------------------------------------------------------- CPU part ----

def test_bf16_rounding():
    x = np.array([1.0, 1 + 2**-8, 1 + 3 * 2**-8, 1 + 2**-9, -3.14159, 0.0, 1e-30], np.float32)
    r = bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie to even (down)
    assert r[2] == 1 + 4 * 2**-8                 # tie to even (up)
    assert r[3] == 1.0
    assert abs(r[4] + 3.140625) < 1e-7 and r[5] == 0.0
    assert np.all(r.view(np.uint32) & 0xFFFF == 0)


def test_model_gradient_matches_finite_differences():
    p = glorot(1)
    X, y = batch(2, 40)
    _, g, _ = forward_backward(p, X, y, pos_weight=3.0, rounded=False)
    rng = np.random.default_rng(3)
    idx = np.concatenate([rng.choice(np.arange(OFF_W1, OFF_B1), 12), rng.choice(np.arange(OFF_W2, OFF_B2), 12),
                          np.arange(OFF_B1, OFF_B1 + 4), np.arange(OFF_B2, OFF_B2 + 4),
                          np.arange(OFF_W3, OFF_W3 + 4), [OFF_B3]])
    h = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (forward_backward(pp, X, y, 3.0, False)[0] - forward_backward(pm, X, y, 3.0, False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7 + 1e-5 * abs(fd), (k, fd, g[k])


def test_rounded_model_close_to_fp64_model():
    p = glorot(4)
    X, y = batch(5, 256)
    l32, g32, _ = forward_backward(p, X, y, rounded=True)
    l64, g64, _ = forward_backward(p, X, y, rounded=False)
    assert abs(l32 - l64) < 2e-2 * abs(l64)
    assert np.linalg.norm(g32 - g64) < 5e-2 * np.linalg.norm(g64)


# ------------------------------------------------------------- GPU part ----

@pytest.mark.gpu
@pytest.mark.parametrize("tc", [True, False], ids=["tcgen05", "mma_sync"])
@pytest.mark.parametrize("n", [1, 63, 64, 127, 128, 200, 4096])
def test_gpu_gradient_matches_numpy(n, tc):
    import gdf
    p = glorot(6).astype(np.float32)
    X, y = batch(7 + n, n)
    m = gdf.Mlp(0)
    m.set_products(tc)
    m.set_params(p)
    assert np.array_equal(m.params(), p)
    g, loss = m.grad(X, y, pos_weight=4.0)
    lr, gr, _ = forward_backward(p, X, y, pos_weight=4.0)
    # accumulation order inside the tensor-core products differs from numpy's,
    # and a BF16 rounding of an intermediate can land one step apart
    assert abs(loss - lr) <= 1e-5 * max(1.0, abs(lr))
    for lo, hi in [(OFF_W1, OFF_B1), (OFF_B1, OFF_W2), (OFF_W2, OFF_B2), (OFF_B2, OFF_W3), (OFF_W3, OFF_B3),
                   (OFF_B3, NPARAM)]:
        err = np.linalg.norm(g[lo:hi] - gr[lo:hi])
        assert err <= 3e-3 * np.linalg.norm(gr[lo:hi]) + 1e-7, (lo, err, np.linalg.norm(gr[lo:hi]))


@pytest.mark.gpu
def test_gpu_predict_matches_numpy():
    import gdf
    p = glorot(8).astype(np.float32)
    X, y = batch(9, 1000)
    m = gdf.Mlp(0)
    m.set_params(p)
    pg = m.predict(X)
    _, _, pr = forward_backward(p, X, y)
    assert np.max(np.abs(pg - pr)) < 2e-3


@pytest.mark.gpu
@pytest.mark.parametrize("tc", [True, False], ids=["tcgen05", "mma_sync"])
def test_gpu_training_learns_a_separable_rule(tc):
    import gdf
    X, y = batch(10, 16384)
    Xt, yt = batch(11, 4096)
    m = gdf.Mlp(3)
    m.set_products(tc)
    acc0 = np.mean((m.predict(Xt) > 0.5) == (yt > 0.5))
    losses = m.train(X, y, epochs=8, batch=512, lr=2e-3, seed=1)
    assert losses[-1] < 0.5 * losses[0]
    acc = np.mean((m.predict(Xt) > 0.5) == (yt > 0.5))
    assert acc > 0.9 and acc > acc0
    # the kernels' gradient at the trained point still matches the restatement
    p = m.params()
    g, _ = m.grad(Xt[:512], yt[:512])
    _, gr, _ = forward_backward(p, Xt[:512], yt[:512])
    assert np.linalg.norm(g - gr) <= 5e-3 * np.linalg.norm(gr)


@pytest.mark.gpu
def test_mlp_argument_errors():
    import gdf
    m = gdf.Mlp(0)
    X, y = batch(0, 10)
    with pytest.raises(gdf.GdfError):
        m.train(X, y, epochs=1, batch=8)          # batch below one 64-sample tile
    with pytest.raises(gdf.GdfError):
        m.grad(X[:0], y[:0])


# ------------------------------------------------- indicator inputs ----

def _basis(x, y):
    return np.array([np.ones_like(x), x, y, x * x - 1 / 3, x * y, y * y - 1 / 3,
                     x ** 3 - 0.6 * x, (x * x - 1 / 3) * y, x * (y * y - 1 / 3), y ** 3 - 0.6 * y])


def features_numpy(uh, gamma):
    """The 90 inputs per interior cell: for the cell and its neighbours E, W,
    N, S, the 6 P2 modes of rho, p and |B|^2 (the latter two projected from
    3x3 Gauss points), scaled by the largest |mean| among the five cells,
    the cell's own mean subtracted from the means, clamped to [-8, 8]."""
    g = np.sqrt(0.6)
    gx, gw = np.array([-g, 0, g]), np.array([5, 8, 5]) / 9
    mm = np.array([1, 1 / 3, 1 / 3, 4 / 45, 1 / 9, 4 / 45])
    ny2, nx2 = uh.shape[2:]
    q = np.zeros((3, 6, ny2, nx2))
    q[0] = uh[0, :6]
    for a in range(3):
        for b in range(3):
            ph = _basis(np.float64(gx[a]), np.float64(gx[b]))
            v = np.einsum("nd...,d->n...", uh, ph)
            rho = v[0]
            b2 = v[5] ** 2 + v[6] ** 2 + v[7] ** 2
            pr = (gamma - 1) * (v[4] - 0.5 * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2) / rho - 0.5 * b2)
            wq = gw[a] * gw[b] * 0.25
            for d in range(6):
                q[1, d] += wq * ph[d] * pr
                q[2, d] += wq * ph[d] * b2
    q[1:] /= mm[None, :, None, None]
    ny, nx = ny2 - 2, nx2 - 2
    sl = [(slice(1, -1), slice(1, -1)), (slice(1, -1), slice(2, None)), (slice(1, -1), slice(0, -2)),
          (slice(2, None), slice(1, -1)), (slice(0, -2), slice(1, -1))]
    F = np.zeros((ny, nx, 5, 3, 6))
    for qq in range(3):
        sc = np.max([np.abs(q[qq, 0][s]) for s in sl], axis=0) + 1e-30
        mc = q[qq, 0][sl[0]]
        for k, s in enumerate(sl):
            v = q[qq][:, s[0], s[1]].copy()
            v[0] -= mc
            F[:, :, k, qq, :] = np.clip(np.moveaxis(v, 0, -1) / sc[..., None], -8, 8)
    return F.reshape(ny * nx, 90)


@pytest.mark.gpu
@pytest.mark.parametrize("problem", ["ot", "blast", "rotor"])
def test_features_match_numpy(problem):
    import gdf
    prob = {"ot": gdf.PROB_ORSZAG_TANG, "blast": gdf.PROB_BLAST, "rotor": gdf.PROB_ROTOR}[problem]
    cfg, _ = gdf.problem_config(prob, 24, 20)
    uh, bx, by = gdf.init_data(cfg, prob)
    s = gdf.Solver(cfg)
    s.upload(uh, bx, by)
    s.prepare()
    uh, _, _ = s.download()
    X = s.features(uh)
    Xr = features_numpy(uh, cfg.gamma)
    assert X.shape == (24 * 20, 90)
    # FP32 on the device: the pressure E - |rho u|^2/2rho - |B|^2/2 cancels a
    # few digits at low plasma beta (blast, rotor), so the bound is absolute
    # on these O(1) scaled inputs
    assert np.max(np.abs(X - Xr)) < 2e-3


# ------------------------------------------------- learned limiter mode ----

def _limit_case(problem, nx, ny, detector, sticky=1):
    import gdf
    from oracle import Oracle
    cfg, _ = gdf.problem_config(problem, nx, ny)
    cfg.detector = detector
    cfg.kxrcf_sticky = sticky
    o = Oracle(cfg)
    uh, bx, by = o.init_data(problem)
    o.set_bc(uh)
    du = o.lh(uh)
    d1, d2 = o.lhez(uh)
    dt = o.dt(uh)
    return cfg, uh + dt * du, bx + dt * d1, by + dt * d2


@pytest.mark.gpu
@pytest.mark.parametrize("problem", [2, 3])   # rotor, blast
def test_learned_mode_reproduces_reference_detectors(problem):
    """t_lo = t_hi = 0: every cell limited, which is the all-cells detector;
    t_lo = 0 < 1 < t_hi: every cell in the uncertain band, where KXRCF (per
    stage, not sticky) decides. Both must match those detectors bit for bit."""
    import gdf
    m = gdf.Mlp(5)
    for (lo, hi), det in [((0.0, 0.0), gdf.DETECT_ALL), ((0.0, 2.0), gdf.DETECT_KXRCF)]:
        cfg, uh, bx, by = _limit_case(problem, 20, 18, gdf.DETECT_LEARNED)
        ref_cfg, _, _, _ = _limit_case(problem, 20, 18, det, sticky=0)
        s = gdf.Solver(cfg)
        s.set_indicator(m, lo, hi)
        ua, ba, ca = uh.copy(), bx.copy(), by.copy()
        fa = s.limit(ua, ba, ca)
        r = gdf.Solver(ref_cfg)
        ub, bb, cb = uh.copy(), bx.copy(), by.copy()
        fb = r.limit(ub, bb, cb)
        assert np.array_equal(ua, ub) and np.array_equal(ba, bb) and np.array_equal(ca, cb), (lo, hi)
        assert np.array_equal(fa & 0xFFFFFF, fb & 0xFFFFFF)


@pytest.mark.gpu
def test_learned_mode_gates_follow_the_network():
    """Thresholds above 1 limit nowhere; the set of gated cells equals the
    cells whose network probability (from gdf_mlp_predict on gdf_features)
    is at least t_hi, away from the decision boundary."""
    import gdf
    cfg, uh, bx, by = _limit_case(3, 24, 24, gdf.DETECT_LEARNED)
    m = gdf.Mlp(7)
    s = gdf.Solver(cfg)
    s.set_indicator(m, 2.0, 2.0)
    f = s.limit(uh.copy(), bx.copy(), by.copy())
    assert not np.any(f & (1 << 24))
    pr = m.predict(s.features(uh)).reshape(24, 24)
    t = float(np.median(pr))
    s.set_indicator(m, t, t)
    f = s.limit(uh.copy(), bx.copy(), by.copy())
    gated = (f & (1 << 24)) != 0
    far = np.abs(pr - t) > 1e-3
    assert np.array_equal(gated[far], (pr >= t)[far])
    assert 0 < gated.sum() < gated.size


@pytest.mark.gpu
def test_learned_mode_needs_a_network():
    import gdf
    cfg, uh, bx, by = _limit_case(2, 16, 16, gdf.DETECT_LEARNED)
    s = gdf.Solver(cfg)
    with pytest.raises(gdf.GdfError):
        s.limit(uh, bx, by)
