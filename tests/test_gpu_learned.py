"""The learned block proposal on the device against the CPU oracle
(oracle/mlp_ref.py), and what the trained network gains.

Tolerances: features |d| <= 1e-3 (asinh of FP32 running sums of up to nharms
unit powers against FP64); network outputs |dz| <= 1e-4 * max|z| and gradients
||dg|| <= 1e-4 * ||g|| (FP32 accumulation against FP64, same BF16 weights);
an Adam step to 1e-6 relative; the BF16 weight copies bit-exact.
"""
import numpy as np
import pytest

from oracle import mlp_ref as m
from tests.fixtures import multi_spectrum, pulsar_spectrum

pytestmark = pytest.mark.gpu


def _cs():
    import cohsearch
    return cohsearch


def _engine(params, amps, N, dt):
    cs = _cs()
    eng = cs.Engine(params)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng


def test_block_features_vs_oracle():
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    dec = cs.decimation_set(32, 4)
    eng = _engine(cs.SearchParams(nharms=32, m=16, decimations=dec), amps, N, dt)
    got = eng.block_features(1.0, 50.0, 100, 2048).cpu().numpy()
    T = N * dt
    lodr = 0.5 / 32
    r_lo = 1.0 * T
    total = int(np.floor((50.0 * T - r_lo) / lodr)) + 1
    want = m.block_features(amps, r_lo, lodr, 2048, total, m.levels_of(32, dec))
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-3


def test_mlp_forward_backward_adam_vs_oracle():
    import torch
    from cohsearch.learned import ProposalMLP
    rng = np.random.default_rng(4)
    x = rng.normal(size=(300, 147)).astype(np.float32)
    y = (rng.random(300) < 0.2).astype(np.float32)
    mlp = ProposalMLP(147, 256, seed=1)
    X = torch.from_numpy(x).cuda()
    p = mlp.params_numpy()
    h1, h2, z = mlp.forward(X)
    rh1, rh2, rz = m.mlp_forward(p, x)
    z = z.cpu().numpy()
    assert np.max(np.abs(z - rz)) <= 1e-4 * np.max(np.abs(rz))
    assert np.max(np.abs(h2.cpu().numpy() - rh2)) <= 1e-4 * np.max(np.abs(rh2))
    loss = float(mlp.loss_and_grads(X, torch.from_numpy(y), 4.0).item())
    rl, rg = m.mlp_backward(p, x, y, 4.0)
    assert loss == pytest.approx(rl, rel=1e-4)
    g = {k: v.cpu().numpy() for k, v in mlp.g.items()}
    for k in rg:
        assert np.linalg.norm(g[k] - rg[k]) <= 1e-4 * np.linalg.norm(rg[k]), k
    # first Adam step: bias-corrected moments give p - lr * g / (|g| + eps)
    lr, eps = 1e-2, 1e-8
    mlp.adam(lr=lr, eps=eps)
    p1 = mlp.params_numpy()
    for k in p:
        want = p[k] - lr * g[k] / (np.abs(g[k]) + eps)
        assert np.allclose(p1[k], want, rtol=1e-6, atol=1e-7), k
    for k in ("w1", "w2", "w3"):
        bits = mlp.bf[k].cpu().numpy().view(np.uint16)
        assert np.array_equal(bits, (m.bf16_round(p1[k]).view(np.uint32) >> 16).astype(np.uint16))


def test_search_blocks_equal_the_full_search():
    cs = _cs()
    from cohsearch import parallel
    amps, N, dt = multi_spectrum()
    dec = cs.decimation_set(32, 4)
    eng = _engine(cs.SearchParams(nharms=32, m=16, decimations=dec, threshold=7.0, synth="fp16"), amps, N, dt)
    full = eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    nb = parallel.band_blocks(N, dt, 0.5, 32, 1.0, 60.0, 100, 2048)
    rng = np.random.default_rng(2)
    hit = np.unique(full["trial"] // 2048)
    sel = np.unique(np.concatenate([hit[::2], rng.choice(nb, 25, replace=False)]))
    got = eng.search_blocks_raw(sel, 1.0, 60.0, 100, 2048, 7.0)
    want = full[np.isin(full["trial"] // 2048, sel)]
    assert len(want) > 0
    assert np.array_equal(got, want)
    assert len(eng.search_blocks_raw([], 1.0, 60.0, 100, 2048, 7.0)) == 0
    with pytest.raises(Exception):
        eng.search_blocks_raw([nb + 3], 1.0, 60.0, 100, 2048, 7.0)


def _labelled(eng, seeds, nsamp, dt, ninj, band):
    import torch
    from cohsearch import FFTFile, learned, synth
    xs, ys = [], []
    for s in seeds:
        rng = np.random.default_rng(s)
        ps = synth.random_pulsars(rng, ninj, 0.1, 750.0, 0.01, 0.20, 6.0, 20.0)
        eng.set_spectrum(FFTFile.from_array(synth.make_spectrum_fd(nsamp, dt, ps, s), nsamp, dt))
        X = eng.block_features(band[0], band[1], 100, 2048)
        raw = eng.search_raw(band[0], band[1], 100, 2048, 8.0)
        xs.append(X)
        ys.append(torch.from_numpy(learned.block_labels(raw, X.shape[0], 2048, 8.0)))
    return torch.cat(xs), torch.cat(ys)


def test_learned_proposal_gains_over_the_full_search():
    """Trained on separately seeded injected spectra (labels: the coherent
    search's own candidates), the network keeps the recall of the full search
    on held-out spectra while re-searching a fraction of the blocks; an
    untrained network needs more blocks at the same validation recall."""
    cs = _cs()
    from cohsearch import FFTFile, learned, synth
    nsamp, dt, band = 1 << 21, 64e-6, (0.1, 125.0)
    eng = cs.Engine(cs.SearchParams(nharms=60, m=16, decimations=cs.decimation_set(60, 6), synth="fp16"))
    Xt, Yt = _labelled(eng, range(100, 130), nsamp, dt, 20, band)
    Xv, Yv = _labelled(eng, range(200, 208), nsamp, dt, 20, band)
    mlp = learned.ProposalMLP(Xt.shape[1], 256, seed=0)
    hist = mlp.fit(Xt, Yt, epochs=20, batch=1024, lr=1e-3)
    assert hist[-1] < hist[0]
    tau = learned.choose_threshold(mlp.scores(Xv), Yv.numpy(), 0.995)
    untrained = learned.ProposalMLP(Xt.shape[1], 256, seed=5)
    tau_u = learned.choose_threshold(untrained.scores(Xv), Yv.numpy(), 0.995)
    rec, frac, frac_u = [], [], []
    for s in (300, 301, 302):
        rng = np.random.default_rng(s)
        ps = synth.random_pulsars(rng, 20, 0.1, 750.0, 0.01, 0.20, 6.0, 20.0)
        eng.set_spectrum(FFTFile.from_array(synth.make_spectrum_fd(nsamp, dt, ps, s), nsamp, dt))
        full = eng.search_raw(band[0], band[1], 100, 2048, 8.0)
        res = learned.learned_search(eng, mlp, tau, band[0], band[1], 100, 2048, 8.0)
        rec.append(learned.recall_of(res.cands, full, 8.0))
        frac.append(len(res.blocks) / res.nblocks)
        frac_u.append(float(np.mean(untrained.scores(eng.block_features(band[0], band[1], 100, 2048)) >= tau_u)))
    print(f"\nlearned proposal: recall {rec}, blocks re-searched {frac} (untrained {frac_u}), loss {hist[0]:.3f}"
          f" -> {hist[-1]:.3f}")
    assert min(rec) >= 0.95
    # the gain over the method without it (the full search: every block) and
    # over the same network untrained
    assert np.mean(frac) < 0.6 and np.mean(frac) < np.mean(frac_u)
