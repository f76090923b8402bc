"""CPU checks of the learned smoother's oracle (oracle/learned.py): H = I - P R annihilates the
fields the coarse grid represents exactly (linear ones), the untrained network (last layer zero)
scores the Jacobi step's loss ||t||^2 / n with no gradient on the hidden layers, and a sample's
target is (H e - omega H q) / s."""
import numpy as np
import torch

from oracle import learned as OL


def test_h_annihilates_linear_fields():
    y, x = np.mgrid[-1:18, -1:18].astype(np.float64)
    c = torch.as_tensor((0.3 * x - 1.7 * y + 2.0)[None])
    assert float(torch.abs(OL.h_apply(c)).max()) < 1e-13
    rng = np.random.default_rng(0)
    r = torch.as_tensor(rng.normal(size=(1, 19, 19)))
    assert float(torch.abs(OL.h_apply(r)).max()) > 0.1


def test_untrained_network_scores_the_jacobi_loss():
    rng = np.random.default_rng(1)
    p = np.zeros(OL.NP, dtype=np.float32)
    p[:432] = rng.normal(0, 0.3, 432)
    p[448:2752] = rng.normal(0, 0.1, 2304)
    inp = OL.to_bf16(rng.uniform(-1, 1, (4, 3, 25, 25)))
    th, te = rng.normal(size=(4, 16, 16)), rng.normal(size=(4, 16, 16))
    nh, ne = np.array([3.0, 1.0, 0.5, 2.0]), np.array([1.0, 2.0, 4.0, 0.5])
    for lam in (0.0, 0.7):
        loss, grad = OL.loss_and_grad(p, inp, th, te, nh, ne, lam)
        want = np.mean([((th[k] ** 2).sum() + lam * (te[k] ** 2).sum()) / (nh[k] + lam * ne[k]) for k in range(4)])
        assert abs(loss - want) <= 1e-12 * want
        assert np.all(grad[:2752] == 0) and np.any(grad[2768:] != 0)


def test_sample_target_definition():
    rng = np.random.default_rng(2)
    N = 65
    q, e = rng.normal(size=(N, N)), rng.normal(size=(N, N))
    vx, vy = rng.normal(size=(N, N)), rng.normal(size=(N, N))
    d = np.abs(rng.normal(size=(N, N))) + 1.0
    inp, th, te, nh, ne = OL.extract(q, e, vx, vy, d, 2.0, 0.8, 0.1, 0.1, 10, 12)
    he = OL.h_apply(torch.as_tensor(e[None, 9:28, 11:30].copy()))[0].numpy()
    hq = OL.h_apply(torch.as_tensor(q[None, 9:28, 11:30].copy()))[0].numpy()
    assert np.allclose(th, (he - 0.8 * hq) / 2.0, rtol=0, atol=1e-14)
    assert np.allclose(te, (e[10:26, 12:28] - 0.8 * q[10:26, 12:28]) / 2.0, rtol=0, atol=1e-14)
    assert abs(nh - (he ** 2).sum() / 4.0) < 1e-12 * nh
    assert abs(ne - (e[10:26, 12:28] ** 2).sum() / 4.0) < 1e-12 * ne
    assert inp.shape == (3, 25, 25) and np.array_equal(inp, OL.to_bf16(inp))
