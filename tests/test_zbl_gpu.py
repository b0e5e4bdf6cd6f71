"""ZBL short-range term (models with ``zbl_enabled = 1``) in the CUDA engine
against the FP64 oracle: global and typewise pair cutoffs, atomic numbers from
the model or from the element symbols, a ZBL outer cutoff beyond the SUS2
cutoff (wider neighbour list), close pairs, weighted backward passes and
batches of cells.  The ZBL pass is FP64 in both engine precisions, so the
SUS2 tolerances apply unchanged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, models, structures  # noqa: E402

E_TOL32, F_RMS32, W_RMS32, TOL64 = 1e-6, 1e-5, 1e-5, 1e-9

CASES = {
    "global": dict(atomic_numbers=[29, 40], inner=1.0, outer=3.0),
    "beyond_rc": dict(atomic_numbers=[29, 40], inner=0.5, outer=5.6),
    "typewise_symbols": dict(factor=1.2, outer=3.5),
    "defaults": dict(atomic_numbers=[29, 40]),
}


def _model(base, model_dir, name):
    return models.add_zbl(base, f"{model_dir}/zbl_{name}.mtp", **CASES[name])


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


def _check(path, box, types, pos, fp64, relative=False):
    """relative=True scales the FP32 bars by the oracle's site-energy, force
    and virial magnitudes (close pairs drive the synthetic SUS2 model far
    below its r_min, to site energies of tens of eV)."""
    orc = O.Oracle(path, symbols=["Cu", "Zr"])
    pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types, pos)
    pot = SUS2_SH(path, types.size, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    pe, f, w = _efs(pot, box, types, pos)
    pot.close()
    if fp64:
        assert np.abs(pe - pe0).max() < TOL64
        assert np.abs(f - f0).max() < 10 * TOL64 * max(1.0, np.abs(f0).max())
        assert np.abs(w - w0).max() < 100 * TOL64 * max(1.0, np.abs(w0).max())
    else:
        es = max(1.0, np.abs(pe0).max()) if relative else 1.0
        fs = max(1.0, np.sqrt((f0 ** 2).mean())) if relative else 1.0
        ws = max(1.0, np.sqrt((w0 ** 2).mean())) if relative else 1.0
        assert np.abs(pe - pe0).max() < E_TOL32 * es
        assert np.sqrt(((f - f0) ** 2).mean()) < F_RMS32 * fs
        assert np.sqrt(((w - w0) ** 2).mean()) < W_RMS32 * ws
    return pe0, f0


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("name", sorted(CASES))
def test_zbl_fcc_matches_oracle(l3k3_path, model_dir, name, fp64):
    path = _model(l3k3_path, model_dir, name)
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.5, 0.5), 0.15, seed=21)
    pe0, _ = _check(path, box, types, pos, fp64)
    # the term is really there: differs from the plain model's energies
    plain = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, pos)[0]
    if name != "defaults":
        assert np.abs(pe0 - plain).max() > 1e-3


@pytest.mark.parametrize("fp64", [False, True])
def test_zbl_close_pairs(l3k3_path, model_dir, fp64):
    # random insertion with pairs down to 1.3 A: strong repulsion
    path = _model(l3k3_path, model_dir, "global")
    box, types, pos = structures.random_insertion(1500, 0.07, 1.3, seed=22)
    pe0, f0 = _check(path, box, types, pos, fp64, relative=True)
    assert np.abs(f0).max() > 10.0


def test_zbl_small_triclinic_cell(l3k3_path, model_dir):
    path = _model(l3k3_path, model_dir, "beyond_rc")
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=23)
    H = box.cpu_h.reshape(3, 3).copy()
    H[0, 1] = 1.3
    from sus2sh import Box
    tri = Box(H.ravel(), box.pbc)
    _check(path, tri, types, pos, fp64=True)


def test_zbl_weighted_backward(l3k3_path, model_dir):
    from sus2sh.autograd import site_energy
    path = _model(l3k3_path, model_dir, "global")
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.15, seed=24)
    N = types.size
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    orc = O.Oracle(path)
    pot = SUS2_SH(path, N, ["Cu", "Zr", "sus2_float=0"])
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev).requires_grad_(True)
    wts = np.random.default_rng(25).normal(size=N)
    e = site_energy(pot, box, t, x)
    (g,) = torch.autograd.grad((e * torch.as_tensor(wts, device=dev)).sum(), x)
    g = g.cpu().numpy().reshape(3, N)
    h = 1e-5
    for i in (0, 11, 50):
        for a in range(3):
            p1 = pos.copy(); p1[a, i] += h
            p2 = pos.copy(); p2[a, i] -= h
            fd = (wts @ orc.efs(box.cpu_h, box.pbc, types, p1)[0]
                  - wts @ orc.efs(box.cpu_h, box.pbc, types, p2)[0]) / (2 * h)
            assert abs(fd - g[a, i]) < 1e-6 * max(1.0, abs(fd))
    pot.close()


@pytest.mark.parametrize("fp64", [False, True])
def test_zbl_batch_of_cells(l3k3_path, model_dir, fp64):
    path = _model(l3k3_path, model_dir, "global")
    off, H, boxes, types, pos = structures.cell_batch(12, 16, 256, dmin=1.4, seed=26)
    N = types.size
    dev = torch.device("cuda")
    pot = SUS2_SH(path, N, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    pe = torch.zeros(N, dtype=torch.float64, device=dev)
    f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
    pot.compute_batch(torch.as_tensor(off, device=dev), torch.as_tensor(H.reshape(-1).copy(), device=dev), t, x,
                      pe, f, w)
    torch.cuda.synchronize()
    assert pot.sync() == 0
    pe, f, w = pe.cpu().numpy(), f.view(3, N).cpu().numpy(), w.view(9, N).cpu().numpy()
    orc = O.Oracle(path)
    etol, ftol = (1e-9, 1e-8) if fp64 else (1e-6, 1e-5)
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        # pairs down to 1.4 A: FP32 bars relative to the site-energy/force scale
        assert np.abs(pe[a:b] - pe0).max() < etol * max(1.0, np.abs(pe0).max())
        assert np.sqrt(((f[:, a:b] - f0) ** 2).mean()) < ftol * max(1.0, np.sqrt((f0 ** 2).mean()))
        assert np.sqrt(((w[:, a:b] - w0) ** 2).mean()) < ftol * max(1.0, np.sqrt((w0 ** 2).mean()))
    pot.close()
