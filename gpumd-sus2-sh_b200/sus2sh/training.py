"""Training-loss gradients through the engine's parameter-gradient C-ABI.

The loss of the energy/force fitting workload,
    L = sum_c (E_c - E_c^t)^2 + lambda_f sum_i |F_i - F_i^t|^2,
over periodic cells c (E_c = sum of the cell's site energies), is evaluated
with sus2sh_compute and differentiated with sus2sh_param_grad, whose force
part is the forward-over-reverse adjoint (see include/sus2sh.h).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .potential import SUS2_SH, Box


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def loss_and_grad(pot: SUS2_SH, cells, targets, force_weight: float = 0.1):
    """cells: list of (Box, types[N], positions[3,N]); targets: list of
    (E_total, F[3,N]).  Returns (L, dL/dmoment_coeffs, dL/dradial_coeffs)."""
    import torch
    info = pot.info()
    nsc = info["scalars"]
    nrad = info["k_max"] * (info["l_max"] + 1) * info["rb_size"]
    dev = torch.device("cuda")
    gw = torch.zeros(nsc, dtype=torch.float64, device=dev)
    gc = torch.zeros(nrad, dtype=torch.float64, device=dev)
    gw_sum = np.zeros(nsc)
    gc_sum = np.zeros(nrad)
    L = 0.0
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = _lib.load()
    for (box, types, pos), (Et, Ft) in zip(cells, targets):
        N = types.size
        t = torch.as_tensor(types.astype(np.int32), device=dev)
        x = torch.as_tensor(np.ascontiguousarray(pos, dtype=np.float64).reshape(-1), device=dev)
        pe = torch.zeros(N, dtype=torch.float64, device=dev)
        f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
        w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
        pot.compute(box, t, x, pe, f, w)
        Ec = float(pe.sum())
        F = f.view(3, N).cpu().numpy()
        dE = Ec - float(Et)
        dF = F - np.asarray(Ft)
        L += dE * dE + force_weight * float((dF * dF).sum())
        ew = torch.full((N,), 2.0 * dE, dtype=torch.float64, device=dev)
        fw = torch.as_tensor((2.0 * force_weight * dF).reshape(-1).copy(), device=dev)
        _lib.check(lib.sus2sh_param_grad(pot.handle, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p),
                                         box.pbc.ctypes.data_as(ctypes.c_void_p), _p(t), _p(x), _p(ew), _p(fw),
                                         _p(gw), _p(gc), stream), "sus2sh_param_grad")
        gw_sum += gw.cpu().numpy()
        gc_sum += gc.cpu().numpy()
    return L, gw_sum, gc_sum
