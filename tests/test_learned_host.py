"""The learned block proposal on the host (no GPU): the oracle's gradients
against finite differences, its features on noise and on an injected pulsar,
the frequency-domain spectrum synthesis, and the label / threshold / recall
helpers of cohsearch.learned."""
import numpy as np
import pytest

from oracle import mlp_ref as m


def _params(rng, din, dh):
    return {"w1": rng.normal(size=(dh, din)).astype(np.float32), "b1": (0.1 * rng.normal(size=dh)).astype(np.float32),
            "w2": rng.normal(size=(dh, dh)).astype(np.float32), "b2": (0.1 * rng.normal(size=dh)).astype(np.float32),
            "w3": rng.normal(size=dh).astype(np.float32), "b3": np.array([0.2], np.float32)}


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng, 6, 5)
    x = rng.normal(size=(9, 6))
    y = (rng.random(9) < 0.4).astype(float)
    loss, g = m.mlp_backward(p, x, y, 3.0, round_weights=False)
    pd = {k: v.astype(np.float64) for k, v in p.items()}
    for k in pd:
        for idx in np.ndindex(pd[k].shape):
            a = {q: v.copy() for q, v in pd.items()}
            b = {q: v.copy() for q, v in pd.items()}
            a[k][idx] += 1e-6
            b[k][idx] -= 1e-6
            fd = (m.bce_loss(m.mlp_forward(a, x, False)[2], y, 3.0) -
                  m.bce_loss(m.mlp_forward(b, x, False)[2], y, 3.0)) / 2e-6
            assert abs(fd - g[k][idx]) < 1e-7
    assert loss == pytest.approx(m.bce_loss(m.mlp_forward(pd, x, False)[2], y, 3.0))


def test_bf16_round_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38], np.float32)
    r = m.bf16_round(x)
    assert list(r[:4]) == [1.0, 1.0, 1.0 + 2 ** -7, -2.5]   # ties to even; exact values kept
    assert np.all(r.view(np.uint32) & 0xFFFF == 0)


def test_features_on_noise_and_an_injected_pulsar():
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "coherentsearch.jl_b200"))
    from cohsearch import synth
    nsamp, dt = 1 << 18, 64e-6
    T = nsamp * dt
    lodr = 0.5 / 16
    r_lo, Nprof = 20.0 * T, 512
    total = int(np.floor((60.0 * T - r_lo) / lodr)) + 1
    lev = m.levels_of(16, [1, 2, 3])
    assert lev == [(1, 16), (2, 8), (3, 5)]
    noise = synth.make_spectrum_fd(nsamp, dt, [], seed=3)
    assert np.mean(np.abs(noise) ** 2) == pytest.approx(1.0, rel=0.02)
    fn = m.block_features(noise, r_lo, lodr, Nprof, total, lev)
    assert fn.shape[1] == 29 and np.median(fn) < 2.5   # asinh(max z) of noise: a few units
    psr = synth.Pulsar(37.0, 0.05, 40.0, 0.3)
    sig = synth.make_spectrum_fd(nsamp, dt, [psr], seed=3)
    fs = m.block_features(sig, r_lo, lodr, Nprof, total, lev)
    b = int((37.0 * T - r_lo) / lodr) // Nprof
    assert fs[b, :16].max() > fn[:, :16].max() + 1.0          # level 1 sees the pulsar's block
    # level 2 at fundamental 37/2 Hz sums harmonics 2, 4, ... of that trial: the pulsar's
    b2 = int((18.5 * T - r_lo) / lodr) // Nprof
    if 0 <= b2 < fs.shape[0]:
        assert fs[b2, 16:24].max() > fn[:, 16:24].max()


def test_labels_threshold_and_recall():
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "coherentsearch.jl_b200"))
    from cohsearch import _lib, learned
    raw = np.zeros(4, _lib.CAND_DTYPE)
    raw["trial"] = [10, 2050, 2060, 9000]
    raw["k"] = [1, 1, 2, 3]
    raw["metric"] = [9.0, 7.5, 12.0, 8.5]
    y = learned.block_labels(raw, 6, 2048, 8.0)
    assert list(y) == [1, 1, 0, 0, 1, 0]
    scores = np.array([0.9, 0.2, 0.1, 0.05, 0.7, 0.3])
    tau = learned.choose_threshold(scores, y, recall=1.0)
    assert np.all(scores[y > 0] >= tau) and tau > 0.19
    assert learned.recall_of(raw[[0, 2]], raw, 8.0) == pytest.approx(2 / 3)
    assert learned.recall_of(raw[:0], raw[:0], 8.0) == 1.0
