"""Real spherical harmonics up to l = 6 (the reference's eval_real_sh and its
solid-harmonic path for l_max > 4, src/force/sus2_sh.cu:2880-3169): the
engine's host build of its device functions and the oracle's closed form
against the complex-harmonic convention, and their gradients against finite
differences.  Also the NVRTC build of the per-edge kernels for shapes without
an ahead-of-time instantiation (no GPU needed to compile)."""
import ctypes

import numpy as np
import pytest

import sus2sh_oracle as O
from sus2sh import _lib

P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731


@pytest.mark.parametrize("L", [0, 1, 2, 3, 4, 5, 6])
def test_engine_harmonics_follow_complex_convention(L):
    lib = _lib.load()
    rng = np.random.default_rng(L)
    for _ in range(40):
        d = rng.normal(size=3)
        u = d / np.linalg.norm(d)
        Y = np.zeros(49)
        assert lib.sus2sh_real_sh(L, *u, P(Y), None, None) == 0
        for l in range(L + 1):
            for m in range(-l, l + 1):
                assert abs(Y[l * l + l + m] - O.real_sh_from_complex(l, m, u)) < 1e-13


@pytest.mark.parametrize("L", [3, 4, 5, 6])
def test_engine_gradient_contraction_is_polynomial_gradient(L):
    # V = sum G_lm grad P_lm(u), P_lm(d) = |d|^l Y_lm(d/|d|) homogeneous
    lib = _lib.load()
    rng = np.random.default_rng(10 + L)

    def poly(d, G):
        r = np.linalg.norm(d)
        Y = np.zeros(49)
        lib.sus2sh_real_sh(L, *(d / r), P(Y), None, None)
        return sum(G[l * l + l + m] * Y[l * l + l + m] * r ** l for l in range(L + 1) for m in range(-l, l + 1))

    for _ in range(20):
        d = rng.normal(size=3)
        u = d / np.linalg.norm(d)
        G = rng.normal(size=49)
        Y, V = np.zeros(49), np.zeros(3)
        assert lib.sus2sh_real_sh(L, *u, P(Y), P(G), P(V)) == 0
        h = 1e-6
        fd = np.array([(poly(u + h * e, G) - poly(u - h * e, G)) / (2 * h) for e in np.eye(3)])
        assert np.abs(fd - V).max() < 1e-7 * max(1.0, np.abs(V).max())


def test_oracle_harmonics_l6_and_gradients():
    lib = ctypes.CDLL(O.build_oracle())
    D = ctypes.c_double
    rng = np.random.default_rng(3)
    for _ in range(30):
        d = rng.normal(size=3) * 1.7
        Y, dY = np.zeros(49), np.zeros(147)
        lib.oracle_real_sh(6, D(d[0]), D(d[1]), D(d[2]), P(Y), P(dY))
        for l in range(7):
            for m in range(-l, l + 1):
                assert abs(Y[l * l + l + m] - O.real_sh_from_complex(l, m, d)) < 1e-13
        h = 1e-6
        for a in range(3):
            e = np.zeros(3)
            e[a] = h
            Yp, Ym = np.zeros(49), np.zeros(49)
            lib.oracle_real_sh(6, *(D(v) for v in d + e), P(Yp), None)
            lib.oracle_real_sh(6, *(D(v) for v in d - e), P(Ym), None)
            assert np.abs((Yp - Ym) / (2 * h) - dY[a::3]).max() < 1e-7


@pytest.mark.parametrize("shape", [(1, 5, 2, 8), (0, 6, 2, 10), (1, 2, 3, 6)])
def test_edge_kernels_compile_with_nvrtc(shape):
    lib = _lib.load()
    rb, rf, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    log = ctypes.create_string_buffer(8192)
    rc = lib.sus2sh_edge_kernel_info(*shape, ctypes.byref(rb), ctypes.byref(rf), ctypes.byref(ms), log, 8192)
    assert rc == 0, lib.sus2sh_last_error().decode()
    assert 0 < rb.value <= 255 and 0 < rf.value <= 255
    assert "sm_100a" in log.value.decode()


@pytest.mark.parametrize("name", ["l3k3", "l4k4"])
def test_model_specialised_edge_kernels_fold_the_coefficients(model_dir, name):
    # the FP32 edge kernels built for one model: every radial coefficient
    # (and derivative-series coefficient) becomes an instruction operand, so
    # the module holds no table in memory and the registers stay within the
    # caps of the parameter-reading build
    from sus2sh import models
    lib = _lib.load()
    path = models.preset_model(name, model_dir)
    info = (ctypes.c_int * 6)()
    log = ctypes.create_string_buffer(1 << 16)
    rc = lib.sus2sh_model_edge_kernel_info(path.encode(), ctypes.cast(info, ctypes.c_void_p), log, 1 << 16)
    assert rc == 0, lib.sus2sh_last_error().decode()
    basic_regs, force_regs, ms, gmem, entries, cubin = list(info)
    kmu_rb = {"l3k3": 12 * 8, "l4k4": 20 * 10}[name]
    assert entries == 2 * kmu_rb  # coefficients, then the derivative series
    assert 0 <= gmem < 4 * entries  # no table in global memory
    assert 0 < basic_regs <= 255 and 0 < force_regs <= 255
    if name == "l3k3":
        assert basic_regs <= 128 and force_regs <= 128
    assert log.value.decode().count("Compiling entry function") == 6
    assert cubin > 0


def test_edge_kernel_shape_limits():
    lib = _lib.load()
    assert lib.sus2sh_edge_kernel_info(1, 7, 1, 8, None, None, None, None, 0) != 0
    assert lib.sus2sh_edge_kernel_info(1, 6, 7, 8, None, None, None, None, 0) != 0  # 7 * 7 > 48 radial functions
    assert lib.sus2sh_edge_kernel_info(1, 3, 3, 17, None, None, None, None, 0) != 0
