"""CPU checks of the learned-proposal restatement (oracle/proposal.py): its backpropagated
gradient equals finite differences of its loss, BF16 rounding is round-to-nearest-even, and the
loss is minimised by bin probabilities proportional to the per-bin weight mass."""
import numpy as np

from nociwick import synthetic as sy
from oracle import proposal as PR


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.1415926], np.float32)
    r = PR.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0          # tie to even (down)
    assert r[2] == 1.0 + 2 ** -7                 # above the tie: up
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12


def test_gradient_matches_finite_differences():
    basis = sy.sd_basis(6, 2, 2, 2)
    nref, nmo = 2, 6
    din, nout = 32, nref * PR.RANK_BINS
    det_bin, sizes = PR.bins(basis, nref)
    rng = np.random.default_rng(0)
    npar = 128 * din + 128 + 128 * 128 + 128 + nout * 128 + nout
    params = rng.normal(0, 0.1, npar)
    rows = rng.integers(0, basis.shape[0], 40)
    mask = PR.valid_mask(det_bin, sizes, rows)
    tbin = det_bin[rng.integers(0, basis.shape[0], 40)]
    tbin = np.where(mask[np.arange(40), tbin], tbin, det_bin[rows] ^ 0)   # keep targets valid
    tbin = np.array([t if mask[i, t] else np.nonzero(mask[i])[0][0] for i, t in enumerate(tbin)])
    w = rng.uniform(0.1, 2.0, 40)
    x = PR.features(basis, rows, nref, nmo, din)
    loss, g = PR.loss_grad(params, x, mask, tbin, w, din, nout, round_bf16=False)
    for k in rng.choice(npar, 60, replace=False):
        e = np.zeros(npar)
        e[k] = 1e-6
        lp, _ = PR.loss_grad(params + e, x, mask, tbin, w, din, nout, round_bf16=False)
        lm, _ = PR.loss_grad(params - e, x, mask, tbin, w, din, nout, round_bf16=False)
        assert abs((lp - lm) / 2e-6 - g[k]) <= 1e-6 + 1e-5 * abs(g[k])


def test_cross_entropy_minimiser_is_the_mass_distribution():
    # for one parent: minimising -sum_b m_b log p_b over the simplex gives p = m / sum m
    m = np.array([0.5, 3.0, 0.0, 1.5])
    z = np.zeros(4)
    mask = (m > 0)[None, :] | np.array([[True, True, True, True]])
    for _ in range(3000):
        p = PR.probs(z[None, :], mask)[0]
        z -= 0.5 * (p * m.sum() - m)
    assert np.allclose(PR.probs(z[None, :], mask)[0], m / m.sum(), atol=1e-3)
