"""Minimal NVE velocity-Verlet driver around the engine, standing in for
GPUMD's integrator (not vendored by the reference) in the benchmark; its
kernels are in libsus2sh_tools.so.

All state is device-resident (torch CUDA tensors, GPUMD SoA layouts); each
step is kick+drift (which also zeroes the force/energy/virial accumulators),
one ``SUS2_SH.compute`` and a kick.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .potential import SUS2_SH, Box


class NVE:
    def __init__(self, potential: SUS2_SH, box: Box, types, positions, velocities, masses, dt_fs: float,
                 device="cuda"):
        import torch
        self.torch = torch
        self.pot = potential
        self.box = box
        self.dt = float(dt_fs)
        self.N = int(types.shape[0])
        dev = torch.device(device)
        self.type = torch.as_tensor(np.ascontiguousarray(types, dtype=np.int32), device=dev)
        self.pos = torch.as_tensor(np.ascontiguousarray(positions, dtype=np.float64).reshape(-1), device=dev)
        self.vel = torch.as_tensor(np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1), device=dev)
        self.inv_mass = torch.as_tensor(1.0 / np.asarray(masses, dtype=np.float64), device=dev)
        self.pe = torch.zeros(self.N, dtype=torch.float64, device=dev)
        self.force = torch.zeros(3 * self.N, dtype=torch.float64, device=dev)
        self.virial = torch.zeros(9 * self.N, dtype=torch.float64, device=dev)
        self.lib = _lib.load_tools()
        self.kernel_launches_per_step = None

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def initial_force(self):
        self.pe.zero_()
        self.force.zero_()
        self.virial.zero_()
        self.pot.compute(self.box, self.type, self.pos, self.pe, self.force, self.virial)

    def step(self):
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        s = self._stream()
        _lib.check_tools(self.lib.sus2sh_md_kick_drift(self.N, self.dt, p(self.inv_mass), p(self.type), p(self.force),
                                                 p(self.vel), p(self.pos), p(self.pe), p(self.virial), s),
                   "md kick_drift")
        self.pot.compute(self.box, self.type, self.pos, self.pe, self.force, self.virial)
        _lib.check_tools(self.lib.sus2sh_md_kick(self.N, self.dt, p(self.inv_mass), p(self.type), p(self.force),
                                           p(self.vel), s), "md kick")

    def kinetic_energy(self) -> float:
        m = 1.0 / self.inv_mass[self.type.long()]
        v = self.vel.view(3, self.N)
        return float(0.5 * (m * (v * v).sum(0)).sum() / 9.648533212331002e-3)
