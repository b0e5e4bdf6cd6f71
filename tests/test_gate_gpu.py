"""Two-layer mu-body gate models (mu-scalar-full and mu-body-linear-combo,
neighbour site mode) in the CUDA engine against the FP64 oracle: energies,
forces and virials in both engine precisions, a shape compiled with NVRTC,
weighted backward passes against finite differences, batches of cells, and
the gate combined with ZBL."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, _lib, models, structures  # noqa: E402

MODES = ["mu-scalar-full", "mu-body-linear-combo"]


def _gate(base, model_dir, mode, tag="l3k3"):
    path = os.path.join(model_dir, f"gate_{tag}_{mode}.mtp")
    if not os.path.exists(path):
        models.add_gate(base, path, mode=mode, seed=31, additive=[1.0, 0.7])
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


def _check(path, box, types, pos, fp64, species=("Cu", "Zr")):
    pot = SUS2_SH(path, types.size, [*species] + (["sus2_float=0"] if fp64 else []))
    assert pot.info()["gate_mode"] in (1, 2)
    pe, f, w = _efs(pot, box, types, pos)
    pot.close()
    pe0, f0, w0 = O.Oracle(path, symbols=list(species)).efs(box.cpu_h, box.pbc, types, pos)
    if fp64:
        assert np.abs(pe - pe0).max() < 1e-9 * max(1.0, np.abs(pe0).max())
        assert np.abs(f - f0).max() < 1e-8 * max(1.0, np.abs(f0).max())
        assert np.abs(w - w0).max() < 1e-7 * max(1.0, np.abs(w0).max())
    else:
        assert np.abs(pe - pe0).max() < 1e-6 * max(1.0, np.abs(pe0).max())
        assert np.sqrt(((f - f0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((f0 ** 2).mean()))
        assert np.sqrt(((w - w0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((w0 ** 2).mean()))
    return pe0, f0


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("mode", MODES)
def test_gate_matches_oracle(l3k3_path, model_dir, mode, fp64):
    path = _gate(l3k3_path, model_dir, mode)
    box, types, pos = structures.fcc(5, 5, 5, 3.8, (0.5, 0.5), 0.1, seed=32)
    _, f0 = _check(path, box, types, pos, fp64)
    # the gate really acts: forces differ from the ungated model's
    f_plain = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, pos)[1]
    assert np.abs(f0 - f_plain).max() > 1e-3


@pytest.mark.parametrize("mode", MODES)
def test_gate_on_nvrtc_shape(model_dir, mode):
    base = os.path.join(model_dir, "gate_base_l2k3r6.mtp")
    if not os.path.exists(base):
        models.write_model(base, l_max=2, k_max=3, body_order=4, rb_size=6, seed=33)
    path = _gate(base, model_dir, mode, tag="l2k3r6")
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.1, seed=34)
    pot = SUS2_SH(path, types.size, ["Cu", "Zr"])
    assert pot.info()["edge_jit"] == 1
    pot.close()
    _check(path, box, types, pos, fp64=False)
    _check(path, box, types, pos, fp64=True)


@pytest.mark.parametrize("mode", MODES)
def test_gate_weighted_backward(l3k3_path, model_dir, mode):
    from sus2sh.autograd import site_energy
    path = _gate(l3k3_path, model_dir, mode)
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=35)
    N = types.size
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    orc = O.Oracle(path)
    pot = SUS2_SH(path, N, ["Cu", "Zr", "sus2_float=0"])
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev).requires_grad_(True)
    wts = np.random.default_rng(36).normal(size=N)
    e = site_energy(pot, box, t, x)
    (g,) = torch.autograd.grad((e * torch.as_tensor(wts, device=dev)).sum(), x)
    g = g.cpu().numpy().reshape(3, N)
    h = 1e-5
    for i in (0, 13, 77):
        for a in range(3):
            p1 = pos.copy(); p1[a, i] += h
            p2 = pos.copy(); p2[a, i] -= h
            fd = (wts @ orc.efs(box.cpu_h, box.pbc, types, p1)[0]
                  - wts @ orc.efs(box.cpu_h, box.pbc, types, p2)[0]) / (2 * h)
            assert abs(fd - g[a, i]) < 1e-6 * max(1.0, abs(fd))
    pot.close()


def test_gate_batch_of_cells(l3k3_path, model_dir):
    path = _gate(l3k3_path, model_dir, "mu-body-linear-combo")
    off, H, boxes, types, pos = structures.cell_batch(8, 16, 200, seed=37)
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


def test_gate_with_zbl(l3k3_path, model_dir):
    gated = _gate(l3k3_path, model_dir, "mu-scalar-full")
    path = models.add_zbl(gated, os.path.join(model_dir, "gate_zbl.mtp"), inner=1.0, outer=3.0)
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.15, seed=38)
    _check(path, box, types, pos, fp64=True)


def test_gate_param_grad_is_reported(l3k3_path, model_dir):
    path = _gate(l3k3_path, model_dir, "mu-scalar-full")
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=39)
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
    assert rc != 0 and "gate" in lib.sus2sh_last_error().decode()
    pot.close()
