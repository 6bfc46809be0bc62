"""GPU tests of the differentiable energy (ewaldcorrel_b200.autograd): the
energy and its gradients dE/dx, dE/dq, dE/dL against the FP64 oracle
(analytic de2/potl outputs and the box adjoint checked by finite differences
in tests/test_cell_adjoint.py), against central finite differences of the
oracle energy (h = 1e-4 nm, FP64), and in batched form on the 64-system
differentiable-batch configuration."""
import numpy as np
import pytest

from ewaldcorrel_b200 import configs
from oracle.oracle import OracleSfac
from tests.spme_testlib import rel_rms
from tests.test_cell_adjoint import cell_gradient

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def oracle_all(L, K, order, x, q, beta, max_m):
    s = OracleSfac(L, np.array(K), order)
    s.set_ewald(beta, max_m)
    s.sfac(q, x)
    vir = np.zeros(6)
    e = s.de1(vir)
    n = len(q)
    dx = np.zeros((n, 3))
    phi = np.zeros(n)
    s.de2(n, q, x, dx)
    s.potl(n, x, phi)
    return e, dx, phi, cell_gradient(L, vir, x, dx)


def oracle_energy(L, K, order, x, q, beta, max_m):
    s = OracleSfac(L, np.array(K), order)
    s.set_ewald(beta, max_m)
    s.sfac(q, x)
    return s.en()


def test_spme_energy_and_gradients_single_system():
    import torch

    from ewaldcorrel_b200.autograd import spme_energy

    rng = np.random.default_rng(12)
    L = np.array([2.4, 2.2, 2.6, 0.3, -0.2, 0.4])
    K, order, beta = (24, 24, 27), 6, 3.2
    max_m = configs.MAX_M_FACTOR * beta
    n = 300
    x = rng.uniform(-1, 4, size=(n, 3))
    q = rng.uniform(-1, 1, n)
    q -= q.mean()
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    qt = torch.tensor(q, device="cuda", requires_grad=True)
    Lt = torch.tensor(L, dtype=torch.float64, requires_grad=True)
    E = spme_energy(xt, qt, Lt, K, order, beta, max_m)
    E.backward()
    e0, dx0, phi0, dL0 = oracle_all(L, K, order, x, q, beta, max_m)
    assert abs(E.item() - e0) <= 1e-6 * abs(e0)
    assert rel_rms(xt.grad.cpu().numpy(), dx0) <= 1e-5
    assert rel_rms(qt.grad.cpu().numpy(), phi0) <= 1e-5
    assert np.abs(Lt.grad.numpy() - dL0).max() <= 1e-5 * np.abs(dL0).max()

    # central finite differences of the FP64 oracle energy, h = 1e-4 nm
    h = 1e-4
    fdL = np.array([(oracle_energy(L + h * e, K, order, x, q, beta, max_m)
                     - oracle_energy(L - h * e, K, order, x, q, beta, max_m)) / (2 * h) for e in np.eye(6)])
    assert np.abs(Lt.grad.numpy() - fdL).max() <= 1e-4 * np.abs(fdL).max()
    for a in (0, 17, 123):
        for c in range(3):
            xp = x.copy(); xp[a, c] += h
            xm = x.copy(); xm[a, c] -= h
            fd = (oracle_energy(L, K, order, xp, q, beta, max_m) - oracle_energy(L, K, order, xm, q, beta, max_m)) / (2 * h)
            assert abs(xt.grad[a, c].item() - fd) <= 1e-4 * np.abs(dx0).max()
    for a in (3, 200):
        qp = q.copy(); qp[a] += h
        qm = q.copy(); qm[a] -= h
        fd = (oracle_energy(L, K, order, x, qp, beta, max_m) - oracle_energy(L, K, order, x, qm, beta, max_m)) / (2 * h)
        assert abs(qt.grad[a].item() - fd) <= 1e-4 * np.abs(phi0).max()


def test_spme_energy_repeat_and_box_change():
    """Same plan reused: a second call and a call after a box change agree
    with the oracle (the plan's graph is re-captured on the box change)."""
    import torch

    from ewaldcorrel_b200.autograd import spme_energy

    rng = np.random.default_rng(3)
    K, order, beta = (24, 24, 24), 4, 3.47
    max_m = configs.MAX_M_FACTOR * beta
    n = 500
    x = rng.uniform(0, 2.5, size=(n, 3))
    q = rng.uniform(-1, 1, n)
    for L in (np.array([2.5, 2.5, 2.5, 0, 0, 0.0]), np.array([2.5, 2.5, 2.5, 0, 0, 0.0]),
              np.array([2.6, 2.4, 2.5, 0.1, 0.0, -0.1])):
        E = spme_energy(torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda"), torch.tensor(L), K, order, beta,
                        max_m)
        e0 = oracle_energy(L, K, order, x, q, beta, max_m)
        assert abs(E.item() - e0) <= 1e-6 * abs(e0)


def test_batch_of_64_systems():
    """The differentiable-batch configuration: 64 systems (64-2048 atoms,
    24^3-48^3 grids, order 4) in one call; energies and all gradients per
    system against the oracle."""
    import torch

    from ewaldcorrel_b200.autograd import SpmeBatch

    systems = configs.cfg4_batch()
    batch = SpmeBatch([(s.n, s.K, s.order, s.beta, s.max_m) for s in systems])
    x = torch.tensor(np.concatenate([s.x for s in systems]), device="cuda", requires_grad=True)
    q = torch.tensor(np.concatenate([s.q for s in systems]), device="cuda", requires_grad=True)
    L = torch.tensor(np.stack([s.L for s in systems]), requires_grad=True)
    E = batch(x, q, L)
    weights = torch.linspace(0.5, 1.5, len(systems), dtype=torch.float64, device="cuda")
    (E * weights).sum().backward()
    gx = x.grad.cpu().numpy()
    gq = q.grad.cpu().numpy()
    gL = L.grad.numpy()
    w = weights.cpu().numpy()
    off = 0
    for i in list(range(0, 64, 9)) + [63]:
        s = systems[i]
        off = batch.offsets[i]
        e0, dx0, phi0, dL0 = oracle_all(s.L, s.K, s.order, s.x, s.q, s.beta, s.max_m)
        assert abs(E[i].item() - e0) <= 1e-6 * abs(e0), i
        assert rel_rms(gx[off:off + s.n] / w[i], dx0) <= 1e-5, i
        assert rel_rms(gq[off:off + s.n] / w[i], phi0) <= 1e-5, i
        assert np.abs(gL[i] / w[i] - dL0).max() <= 1e-5 * np.abs(dL0).max(), i
