"""CPU check of the box derivative used by the autograd path: at fixed
Cartesian positions, dE/dL = lower(-V iL^T Pi - sum_a s_a (dE/dx_a)^T), with
Pi the virial de1 returns (sfac.cpp:384-390) and s_a = iL^T x_a unwrapped.
Pinned against central finite differences of the FP64 oracle energy."""
import numpy as np

from oracle.oracle import LofS, OracleSfac, SofL


def cell_gradient(L, vir, x, dx):
    V = L[0] * L[1] * L[2]
    iL = np.linalg.inv(LofS(L))
    Pi = np.array([[vir[0], vir[3], vir[4]], [vir[3], vir[1], vir[5]], [vir[4], vir[5], vir[2]]])
    D = -V * iL.T @ Pi - (x @ iL).T @ dx
    return SofL(D)


def test_cell_adjoint_matches_finite_differences(oracle_built):
    rng = np.random.default_rng(4)
    L = np.array([2.1, 2.3, 1.9, 0.4, -0.3, 0.2])
    K, order, beta, max_m = (20, 24, 18), 4, 3.0, 6.0
    n = 60
    x = rng.uniform(-1, 3, size=(n, 3))
    q = rng.uniform(-1, 1, n)
    q -= q.mean()

    def energy(L6):
        s = OracleSfac(L6, np.array(K), order)
        s.set_ewald(beta, max_m)
        s.sfac(q, x)
        return s.en()

    s = OracleSfac(L, np.array(K), order)
    s.set_ewald(beta, max_m)
    s.sfac(q, x)
    vir = np.zeros(6)
    s.de1(vir)
    dx = np.zeros((n, 3))
    s.de2(n, q, x, dx)
    ana = cell_gradient(L, vir, x, dx)
    h = 1e-5
    fd = np.array([(energy(L + h * e) - energy(L - h * e)) / (2 * h) for e in np.eye(6)])
    assert np.abs(ana - fd).max() <= 1e-8 * np.abs(fd).max()
