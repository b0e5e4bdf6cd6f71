"""Parameter gradients of the energy/force loss (forward-over-reverse force
term) against central finite differences of the FP64 oracle's loss.

Loss of the fitting workload: L = sum_c (E_c - E_t)^2 + 0.1 sum |F - F_t|^2
over 64 FCC cells of 108 atoms, targets from a second seeded model, gradients
with respect to the linear weights (moment_coeffs) and radial coefficients
(16 of each sampled), FD step 1e-4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, models, structures  # noqa: E402
from sus2sh.training import loss_and_grad  # noqa: E402

H = 1e-4


def _cells(n, seed):
    return [structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=seed + c) for c in range(n)]


def _oracle_loss(orc, cells, targets):
    L = 0.0
    for (box, types, pos), (Et, Ft) in zip(cells, targets):
        pe, f, _ = orc.efs(box.cpu_h, box.pbc, types, pos)
        L += (pe.sum() - Et) ** 2 + 0.1 * ((f - Ft) ** 2).sum()
    return L


@pytest.fixture(scope="module")
def setup(model_dir):
    path = models.preset_model("l3k3", model_dir)
    tpath = models.preset_model("l3k3_target", model_dir)
    cells = _cells(64, 300)  # the fitting workload: 64 cells of 108 atoms
    torc = O.Oracle(tpath)
    targets = []
    for box, types, pos in cells:
        pe, f, _ = torc.efs(box.cpu_h, box.pbc, types, pos)
        targets.append((pe.sum(), f))
    return path, cells, targets


@pytest.mark.parametrize("fp64", [True, False])
def test_param_grad_matches_finite_differences(setup, fp64):
    path, cells, targets = setup
    pot = SUS2_SH(path, cells[0][1].size, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    L, gw, gc = loss_and_grad(pot, cells, targets)
    orc = O.Oracle(path)
    L0 = _oracle_loss(orc, cells, targets)
    assert abs(L - L0) < (1e-9 if fp64 else 1e-5) * max(1.0, abs(L0))
    rng = np.random.default_rng(5)
    ws = rng.choice(gw.size, 16, replace=False)
    cs = rng.choice(gc.size, 16, replace=False)
    rel = 1e-5 if fp64 else 2e-3
    for kind, idxs, g, arr in (("w", ws, gw, orc.arrays.w), ("c", cs, gc, orc.arrays.radial)):
        scale = np.abs(g).max()
        for q in idxs:
            old = arr[q]
            arr[q] = old + H
            Lp = _oracle_loss(orc, cells, targets)
            arr[q] = old - H
            Lm = _oracle_loss(orc, cells, targets)
            arr[q] = old
            fd = (Lp - Lm) / (2 * H)
            assert abs(fd - g[q]) < rel * scale + 1e-7, (kind, q, fd, g[q], scale)
    pot.close()


@pytest.mark.parametrize("fp64", [True, False])
def test_generated_and_interpreted_products_agree(setup, fp64):
    # the model-specialised forward-over-reverse product kernel (default) and
    # the flat-product interpreter (sus2_sh_cg_jit=0, used for graphs above the
    # straight-line size) give the same gradients
    path, cells, targets = setup
    opts = ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else [])
    pot = SUS2_SH(path, cells[0][1].size, opts)
    L1, gw1, gc1 = loss_and_grad(pot, cells, targets)
    pot.close()
    pot = SUS2_SH(path, cells[0][1].size, opts + ["sus2_sh_cg_jit=0"])
    L2, gw2, gc2 = loss_and_grad(pot, cells, targets)
    pot.close()
    tol = 1e-10 if fp64 else 2e-5
    assert abs(L1 - L2) <= tol * max(1.0, abs(L2))
    assert np.abs(gw1 - gw2).max() <= tol * np.abs(gw2).max()
    assert np.abs(gc1 - gc2).max() <= tol * np.abs(gc2).max()


def test_energy_only_gradient_is_moment_sum(setup):
    # with force_weight = 0 and unit energy weights, dL/dw_s = sum_i c_t M_i[s]:
    # compare against the oracle's moments through the linear structure of E
    path, cells, _ = setup
    box, types, pos = cells[0]
    N = types.size
    pot = SUS2_SH(path, N, ["Cu", "Zr", "sus2_float=0"])
    import ctypes
    from sus2sh import _lib
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    ew = torch.ones(N, dtype=torch.float64, device=dev)
    info = pot.info()
    gw = torch.zeros(info["scalars"], dtype=torch.float64, device=dev)
    gc = torch.zeros(info["k_max"] * (info["l_max"] + 1) * info["rb_size"], dtype=torch.float64, device=dev)
    p = lambda a: ctypes.c_void_p(a.data_ptr())
    lib = _lib.load()
    rc = lib.sus2sh_param_grad(pot.handle, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p),
                               box.pbc.ctypes.data_as(ctypes.c_void_p), p(t), p(x), p(ew), None, p(gw), p(gc),
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    # E_tot is linear in w: E_tot(w) = E_tot(0) + sum_s w_s dE/dw_s
    orc = O.Oracle(path)
    pe, _, _ = orc.efs(box.cpu_h, box.pbc, types, pos)
    w0 = orc.arrays.w.copy()
    orc.arrays.w[:] = 0.0
    pe0, _, _ = orc.efs(box.cpu_h, box.pbc, types, pos)
    orc.arrays.w[:] = w0
    assert abs((pe.sum() - pe0.sum()) - float(gw.cpu().numpy() @ w0)) < 1e-9 * max(1.0, abs(pe.sum()))
    pot.close()
