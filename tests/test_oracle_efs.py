"""Self-consistency of the FP64 oracle: C vs independent pure-Python
evaluator, forces vs finite differences of the energy, invariances and the
virial identity, on the Chebyshev-sss and the Laguerre-log1p radial bases.
(The oracle's energies and forces are also compared with the reference's own
engine on the GPU, tests/test_ref_parity_gpu.py.)"""
import numpy as np
import pytest

import sus2sh_oracle as O
from sus2sh import structures
from sus2sh_graph import load_mtp


@pytest.fixture(scope="module", params=["chebyshev_sss", "laguerre_log1p"])
def orc(request, l3k3_path, laguerre_path):
    return O.Oracle(l3k3_path if request.param == "chebyshev_sss" else laguerre_path)


def test_c_oracle_matches_python_evaluator(orc):
    box, types, pos = structures.fcc(1, 1, 1, 3.8, (0.5, 0.5), 0.08, seed=3)
    pe, f, v = orc.efs(box.cpu_h, box.pbc, types, pos)
    pe2, f2, v2 = O.python_efs(orc.model, box.cpu_h, box.pbc, types, pos, reach=2)
    assert np.abs(pe - pe2).max() < 1e-10
    assert np.abs(f - f2).max() < 1e-7
    assert np.abs(v - v2).max() < 1e-5 * (1 + np.abs(v).max())


def test_real_harmonics_follow_complex_convention():
    import ctypes
    lib = ctypes.CDLL(O.build_oracle())
    rng = np.random.default_rng(0)
    for _ in range(20):
        d = rng.normal(size=3)
        Y = np.zeros(25)
        lib.oracle_real_sh(4, ctypes.c_double(d[0]), ctypes.c_double(d[1]), ctypes.c_double(d[2]),
                           Y.ctypes.data_as(ctypes.c_void_p), None)
        for l in range(5):
            for m in range(-l, l + 1):
                assert abs(Y[l * l + l + m] - O.real_sh_from_complex(l, m, d)) < 1e-12


def _total_energy(orc, box, types, pos):
    return orc.efs(box.cpu_h, box.pbc, types, pos)[0].sum()


def test_forces_are_minus_energy_gradient(orc):
    box, types, pos = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.1, seed=4)
    pe, f, v = orc.efs(box.cpu_h, box.pbc, types, pos)
    h = 1e-5
    rng = np.random.default_rng(1)
    for i in rng.choice(types.size, 6, replace=False):
        for a in range(3):
            p1 = pos.copy(); p1[a, i] += h
            p2 = pos.copy(); p2[a, i] -= h
            fd = -(_total_energy(orc, box, types, p1) - _total_energy(orc, box, types, p2)) / (2 * h)
            assert abs(fd - f[a, i]) < 1e-7 * max(1.0, abs(f[a, i]))


def test_virial_matches_strain_derivative(orc):
    # sum_i W_i = -dE/d(strain) for a homogeneous deformation of a periodic cell
    box, types, pos = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.1, seed=6)
    pe, f, v = orc.efs(box.cpu_h, box.pbc, types, pos)
    W = v.sum(axis=1)
    full = np.array([[W[0], W[3], W[4]], [W[6], W[1], W[5]], [W[7], W[8], W[2]]])
    H = box.cpu_h.reshape(3, 3)
    h = 1e-6
    for a in range(3):
        for b in range(3):
            eps = np.zeros((3, 3)); eps[a, b] = h
            def energy(e):
                F = np.eye(3) + e
                return _total_energy(orc, type(box)((F @ H).ravel(), box.pbc), types, F @ pos)
            dE = (energy(eps) - energy(-eps)) / (2 * h)
            # W^{ba} = -sum d_b dE_a = -dE/d(eps_ab)
            assert abs(-dE - full[b, a]) < 1e-6 * max(1.0, abs(full[b, a]))


def test_rotation_and_translation_invariance(orc):
    # isolated cluster (no periodicity): E invariant, sum of forces zero
    box, types, pos = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.1, seed=7)
    big = type(box).orthorhombic(200, 200, 200, pbc=(0, 0, 0))
    pos = pos + 50.0
    pe, f, v = orc.efs(big.cpu_h, big.pbc, types, pos)
    assert np.abs(f.sum(axis=1)).max() < 1e-10
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    R = R @ np.array([[1, 0, 0], [0, np.cos(0.3), -np.sin(0.3)], [0, np.sin(0.3), np.cos(0.3)]])
    c = pos.mean(axis=1, keepdims=True)
    pos2 = R @ (pos - c) + c + 3.1
    pe2, f2, _ = orc.efs(big.cpu_h, big.pbc, types, pos2)
    assert np.abs(pe - pe2).max() < 1e-10
    assert np.abs(R @ f - f2).max() < 1e-9


def test_cell_list_matches_brute_force(orc):
    # a 2x2x2-cell crystal (7.6 A box: all-image brute force) tiled 2x2x2 into a
    # 15.2 A box (cell list) gives identical per-atom results
    box1, types1, pos1 = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.1, seed=0)
    pe1, f1, v1 = orc.efs(box1.cpu_h, box1.pbc, types1, pos1)
    L = 7.6
    shifts = [np.array([[x], [y], [z]]) * L for x in (0, 1) for y in (0, 1) for z in (0, 1)]
    pos2 = np.concatenate([pos1 + s for s in shifts], axis=1)
    types2 = np.concatenate([types1] * 8)
    box2 = type(box1).orthorhombic(2 * L, 2 * L, 2 * L)
    pe2, f2, v2 = orc.efs(box2.cpu_h, box2.pbc, types2, pos2)
    n = types1.size
    for k in range(8):
        assert np.abs(pe2[k * n:(k + 1) * n] - pe1).max() < 1e-10
        assert np.abs(f2[:, k * n:(k + 1) * n] - f1).max() < 1e-10
        assert np.abs(v2[:, k * n:(k + 1) * n] - v1).max() < 1e-9
