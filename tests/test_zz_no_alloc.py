"""sus2sh_cg_energy_noalloc: the CG product stage without device allocation.

This entry point serves callers that cannot call cudaMalloc when they need
the contraction (an MD code that holds all device memory in its own fixed
pool and forbids allocation during a run).  It is checked through the C-ABI against the regular entry point
sus2sh_forward on the same structure, on two calls in a row (the second call
reuses the fixed work area the first one left behind), and its adjoints
against the FP64 oracle.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, _lib, structures  # noqa: E402

E_TOL32 = 1e-6   # eV/atom, the FP32 parity bar used throughout the GPU tests
G_TOL32 = 1e-5   # relative to the largest adjoint


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("fp64", [False, True])
def test_noalloc_matches_forward_entry_point(l3k3_path, fp64):
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.05, seed=21)
    N = types.size
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    pe_ref = torch.empty(N, dtype=torch.float64, device=dev)
    pot.forward(box, t, x, pe_ref)                 # existing entry point
    torch.cuda.synchronize()
    pe_ref = pe_ref.cpu().numpy()

    orc = O.Oracle(l3k3_path)
    B = orc.basics(box.cpu_h, box.pbc, types, pos)  # model basic order
    _, G_oracle = orc.cg_energy(types, B)
    dtype = torch.float64 if fp64 else torch.float32
    Bd = torch.as_tensor(B, dtype=dtype, device=dev).contiguous()
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    tol = 1e-9 if fp64 else E_TOL32
    for call in range(2):
        pe = torch.full((N,), np.nan, dtype=torch.float64, device=dev)
        G = torch.full(tuple(B.shape), np.nan, dtype=dtype, device=dev)
        rc = lib.sus2sh_cg_energy_noalloc(pot.handle, N, _ptr(t), _ptr(Bd), _ptr(pe), _ptr(G), stream)
        assert rc == 0, lib.sus2sh_last_error().decode()
        torch.cuda.synchronize()
        de = np.abs(pe.cpu().numpy() - pe_ref).max()
        assert de < tol, (call, de)
        g = G.cpu().numpy().astype(np.float64)
        assert np.abs(g - G_oracle).max() < (1e-10 if fp64 else G_TOL32) * np.abs(G_oracle).max(), call
    pot.close()


def test_noalloc_rejects_sizes_beyond_the_work_area(l3k3_path):
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, 64, ["Cu", "Zr"])
    t = torch.zeros(64, dtype=torch.int32, device=dev)
    B = torch.zeros((48, 64), dtype=torch.float32, device=dev)
    pe = torch.zeros(64, dtype=torch.float64, device=dev)
    G = torch.zeros((48, 64), dtype=torch.float32, device=dev)
    lib = _lib.load()
    # the size check precedes any launch, so the small arrays are never read
    rc = lib.sus2sh_cg_energy_noalloc(pot.handle, 10_000_000, _ptr(t), _ptr(B), _ptr(pe), _ptr(G), None)
    assert rc == -3
    msg = lib.sus2sh_last_error().decode()
    assert "fixed maximum" in msg and "N <=" in msg
    pot.close()


def test_noalloc_marks_unknown_species_with_nan(l3k3_path):
    """An atom whose species lies outside the model gets NaN energy and NaN
    adjoints; the other atoms keep the values of a call without it."""
    box, types, pos = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.05, seed=22)
    N = types.size
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"])
    orc = O.Oracle(l3k3_path)
    B = orc.basics(box.cpu_h, box.pbc, types, pos)
    Bd = torch.as_tensor(B, dtype=torch.float32, device=dev).contiguous()
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = []
    for bad in (None, 5):
        tt = types.copy()
        if bad is not None:
            tt[bad] = 7                      # species_count is 2
        t = torch.as_tensor(tt, device=dev)
        pe = torch.zeros(N, dtype=torch.float64, device=dev)
        G = torch.zeros(tuple(B.shape), dtype=torch.float32, device=dev)
        rc = lib.sus2sh_cg_energy_noalloc(pot.handle, N, _ptr(t), _ptr(Bd), _ptr(pe), _ptr(G), stream)
        assert rc == 0, lib.sus2sh_last_error().decode()
        torch.cuda.synchronize()
        out.append((pe.cpu().numpy(), G.cpu().numpy()))
    (pe0, g0), (pe1, g1) = out
    assert np.isnan(pe1[5]) and np.isnan(g1[:, 5]).all()
    keep = np.arange(N) != 5
    assert np.isfinite(pe1[keep]).all()
    assert np.array_equal(pe1[keep], pe0[keep]) and np.array_equal(g1[:, keep], g0[:, keep])
    pot.close()
