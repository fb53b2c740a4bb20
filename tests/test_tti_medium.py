"""The tilted-VTI medium builder's rotation (ecsg_b200/workloads.py
tti_stiffness, restated on the device in csrc/medium.cu): the Bond-matrix form
agrees with rotating the full fourth-order tensor, the rotated medium keeps the
qP / S moduli along its symmetry axis, and a vertical axis leaves VTI as it is."""
import math

import numpy as np

from ecsg_b200.workloads import VOIGT, bond_matrix, rotation, tti_stiffness, vti_stiffness


def _full(C):
    """Voigt (6, 6) -> fourth-order (3, 3, 3, 3) tensor."""
    idx = {}
    for I, (i, j) in enumerate(VOIGT):
        idx[(i, j)] = idx[(j, i)] = I
    T = np.zeros((3, 3, 3, 3))
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for l in range(3):
                    T[i, j, k, l] = C[idx[(i, j)], idx[(k, l)]]
    return T


def test_bond_matrix_equals_tensor_rotation():
    rng = np.random.default_rng(0)
    for _ in range(20):
        A = rng.standard_normal((6, 6))
        C = A @ A.T + 6 * np.eye(6)
        dip, azi = rng.uniform(0, math.pi), rng.uniform(-math.pi, math.pi)
        a = rotation(np.float64(dip), np.float64(azi))
        M = bond_matrix(a)
        got = _full(M @ C @ M.T)
        want = np.einsum("ip,jq,kr,ls,pqrs->ijkl", a, a, a, a, _full(C))
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
        assert np.allclose(a @ a.T, np.eye(3), atol=1e-15)


def test_symmetry_axis_moduli():
    rng = np.random.default_rng(1)
    vp, vs, rho = 3.0, 1.6, 2.2
    th = (0.10, 0.05, 0.08)
    for _ in range(10):
        dip, azi = rng.uniform(0, math.radians(30)), rng.uniform(-math.pi, math.pi)
        C = tti_stiffness(vp, vs, rho, dip, azi, th)
        n = np.array([math.sin(dip) * math.cos(azi), math.sin(dip) * math.sin(azi), math.cos(dip)])
        G = np.einsum("ijkl,j,l->ik", _full(C), n, n)      # Christoffel matrix
        ev = np.sort(np.linalg.eigvalsh(G))
        assert np.allclose(ev, [rho * vs * vs, rho * vs * vs, rho * vp * vp], rtol=1e-12)
        assert np.allclose(C, C.T, atol=1e-12)
        assert np.linalg.eigvalsh(C).min() > 0


def test_vertical_axis_is_vti():
    C0 = vti_stiffness(3.0, 1.6, 2.2, 0.1, 0.05, 0.08)
    for azi in (0.0, 0.7, -2.0):
        C = tti_stiffness(3.0, 1.6, 2.2, 0.0, azi, (0.1, 0.05, 0.08))
        assert np.abs(C - C0).max() <= 1e-12 * np.abs(C0).max()
