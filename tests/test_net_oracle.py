"""CPU pin of the network oracle: its analytic gradients equal central finite differences."""
import numpy as np

import ewg


def _random_params(rng):
    p = np.zeros(sum(27 * co * ci + co for ci, co in zip(ewg.NET_CIN, ewg.NET_COUT)))
    for (w, b, ci, co), cir, cor in zip(ewg.net_layout(), ewg.NET_CIN_REAL, ewg.NET_COUT_REAL):
        W = np.zeros((27, co, ci))
        W[:, :cor, :cir] = rng.normal(0, 0.3, size=(27, cor, cir))
        p[w:b] = W.ravel()
        p[b:b + cor] = rng.normal(0, 0.1, size=cor)
    return p


def test_oracle_gradients_match_finite_differences():
    import net_oracle
    rng = np.random.default_rng(0)
    p = _random_params(rng)
    f = rng.normal(size=(1, 3, 4, 5, 5))
    t = rng.normal(size=(1, 3, 4, 5, 2))
    loss, y, g = net_oracle.loss_and_grads(p, f, t)
    nz = np.flatnonzero(g)
    idx = rng.choice(nz, size=40, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (net_oracle.loss_and_grads(pp, f, t)[0] - net_oracle.loss_and_grads(pm, f, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])
