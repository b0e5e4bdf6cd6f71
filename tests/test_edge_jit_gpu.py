"""Model shapes without an ahead-of-time edge-kernel build (sh_l_max 5 and 6
on the reference's solid-harmonic path, and uncommon (L, K, rb) shapes): the
edge kernels come from NVRTC at load, the results must match the FP64 oracle
like the precompiled shapes do.  Forcing the NVRTC build on a precompiled
shape must reproduce the ahead-of-time kernels, and so must the FP32 build
specialised to a model's radial coefficients (the default for FP32 models)."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, _lib, models, structures  # noqa: E402

SHAPES = {
    "l5k2b4": dict(l_max=5, k_max=2, body_order=4, rb_size=8, seed=51),
    "l6k2b3": dict(l_max=6, k_max=2, body_order=3, rb_size=10, seed=61),
    "l2k3b4r6": dict(l_max=2, k_max=3, body_order=4, rb_size=6, seed=21),
}


def _model(model_dir, name):
    path = os.path.join(model_dir, f"jit_{name}.mtp")
    if not os.path.exists(path):
        models.write_model(path, **SHAPES[name])
    return path


def _efs(pot, box, types, pos):
    N = types.size
    dev = torch.device("cuda")
    t = torch.as_tensor(types.astype(np.int32), device=dev)
    x = torch.as_tensor(np.ascontiguousarray(pos).reshape(-1), device=dev)
    pe = torch.zeros(N, dtype=torch.float64, device=dev)
    f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
    pot.compute(box, t, x, pe, f, w)
    torch.cuda.synchronize()
    assert pot.sync() == 0
    return pe.cpu().numpy(), f.cpu().numpy().reshape(3, N), w.cpu().numpy().reshape(9, N)


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("name", sorted(SHAPES))
def test_nvrtc_shapes_match_oracle(model_dir, name, fp64):
    path = _model(model_dir, name)
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.1, seed=70)
    pot = SUS2_SH(path, types.size, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    info = pot.info()
    # FP32: the build specialised to the model; FP64: the build of the shape
    assert info["edge_jit"] == (1 if fp64 else 2) and info["edge_jit_force_registers"] > 0
    pe, f, w = _efs(pot, box, types, pos)
    pot.close()
    pe0, f0, w0 = O.Oracle(path).efs(box.cpu_h, box.pbc, types, pos)
    if fp64:
        assert np.abs(pe - pe0).max() < 1e-9 * max(1.0, np.abs(pe0).max())
        assert np.abs(f - f0).max() < 1e-8 * max(1.0, np.abs(f0).max())
        assert np.abs(w - w0).max() < 1e-7 * max(1.0, np.abs(w0).max())
    else:
        assert np.abs(pe - pe0).max() < 1e-6 * max(1.0, np.abs(pe0).max())
        assert np.sqrt(((f - f0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((f0 ** 2).mean()))
        assert np.sqrt(((w - w0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((w0 ** 2).mean()))


@pytest.mark.parametrize("fp64", [False, True])
def test_forced_nvrtc_build_reproduces_precompiled_kernels(l3k3_path, fp64):
    box, types, pos = structures.fcc(5, 5, 5, 3.8, (0.5, 0.5), 0.1, seed=71)
    opts = ["Cu", "Zr", "sus2_sh_autotune=0", "sus2_sh_model_edges=0"] + (["sus2_float=0"] if fp64 else [])
    a = SUS2_SH(l3k3_path, types.size, opts)
    assert a.info()["edge_jit"] == 0
    ra = _efs(a, box, types, pos)
    a.close()
    b = SUS2_SH(l3k3_path, types.size, opts + ["sus2_sh_edge_jit=1"])
    assert b.info()["edge_jit"] == 1
    rb = _efs(b, box, types, pos)
    b.close()
    tol = 1e-12 if fp64 else 1e-6
    for x, y in zip(ra, rb):
        assert np.abs(x - y).max() <= tol * max(1.0, np.abs(x).max())


@pytest.mark.parametrize("autotune", [0, 1])
def test_model_specialised_kernels_reproduce_parameter_kernels(l3k3_path, autotune):
    # the same FP32 arithmetic with each radial coefficient an immediate
    # operand instead of a kernel-parameter load; with the tile autotuner on,
    # every CTA size of the specialised build may be picked
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.64, 0.36), 0.08, seed=74)
    opts = ["Cu", "Zr", f"sus2_sh_autotune={autotune}"]
    a = SUS2_SH(l3k3_path, types.size, opts + ["sus2_sh_model_edges=0"])
    ra = _efs(a, box, types, pos)
    assert a.info()["edge_jit"] == 0
    a.close()
    b = SUS2_SH(l3k3_path, types.size, opts)
    rb = _efs(b, box, types, pos)
    info = b.info()
    b.close()
    assert info["edge_jit"] == 2 and info["force_block"] in (64, 128, 256)
    for x, y in zip(ra, rb):
        assert np.abs(x - y).max() <= 1e-6 * max(1.0, np.abs(x).max())


def test_model_specialised_kernels_large_model(l4k4_path):
    # L=4 K=4 rb=10 rational three-species model through the specialised build
    box, types, pos = structures.random_insertion(400, 0.06, 2.1, (1.0, 1.0, 1.0), (0.5, 0.35, 0.15), seed=75)
    pot = SUS2_SH(l4k4_path, types.size, ["Cu", "Zr", "Al"])
    assert pot.info()["edge_jit"] == 2
    pe, f, w = _efs(pot, box, types, pos)
    pot.close()
    pe0, f0, w0 = O.Oracle(l4k4_path).efs(box.cpu_h, box.pbc, types, pos)
    assert np.abs(pe - pe0).max() < 5e-6 * max(1.0, np.abs(pe0).max())
    assert np.sqrt(((f - f0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((f0 ** 2).mean()))
    assert np.sqrt(((w - w0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((w0 ** 2).mean()))


def test_nvrtc_shape_in_a_batch_of_cells(model_dir):
    path = _model(model_dir, "l5k2b4")
    off, H, boxes, types, pos = structures.cell_batch(6, 16, 128, seed=72)
    N = types.size
    dev = torch.device("cuda")
    pot = SUS2_SH(path, N, ["Cu", "Zr", "sus2_float=0"])
    pe = torch.zeros(N, dtype=torch.float64, device=dev)
    f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
    pot.compute_batch(torch.as_tensor(off, device=dev), torch.as_tensor(H.reshape(-1).copy(), device=dev),
                      torch.as_tensor(types, device=dev), torch.as_tensor(pos.reshape(-1).copy(), device=dev),
                      pe, f, w)
    torch.cuda.synchronize()
    assert pot.sync() == 0
    pe, f = pe.cpu().numpy(), f.view(3, N).cpu().numpy()
    orc = O.Oracle(path)
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        pe0, f0, _ = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        assert np.abs(pe[a:b] - pe0).max() < 1e-9 * max(1.0, np.abs(pe0).max())
        assert np.abs(f[:, a:b] - f0).max() < 1e-8 * max(1.0, np.abs(f0).max())
    pot.close()


def test_param_grad_on_nvrtc_shape_is_reported(model_dir):
    path = _model(model_dir, "l6k2b3")
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=73)
    N = types.size
    pot = SUS2_SH(path, N, ["Cu", "Zr"])
    dev = torch.device("cuda")
    p = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    ew = torch.ones(N, dtype=torch.float64, device=dev)
    gw = torch.zeros(1024, dtype=torch.float64, device=dev)
    gc = torch.zeros(4096, dtype=torch.float64, device=dev)
    lib = _lib.load()
    rc = lib.sus2sh_param_grad(pot.handle, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p),
                               box.pbc.ctypes.data_as(ctypes.c_void_p), p(t), p(x), p(ew), None, p(gw), p(gc),
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc != 0 and "ahead of time" in lib.sus2sh_last_error().decode()
    pot.close()
