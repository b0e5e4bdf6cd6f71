"""Host-side mirror of the reference's GPUMD plugin class.

``SUS2_SH`` has the constructor and ``compute`` of ``class SUS2_SH : public
Potential`` (src/force/sus2_sh.cuh:7-25): it takes the model file, the atom
count and the run.in option tokens (element symbols first), and ``compute``
accumulates per-atom energy, SoA forces and the 9-component per-atom virial
into caller-owned device arrays, exactly as GPUMD's ``Force::compute`` expects
(src/force/force.cu:492-540).  Device arrays are torch CUDA tensors standing in
for GPUMD's ``GPU_Vector``; every call goes through the C-ABI in
include/sus2sh.h.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

MODEL_INFO_FIELDS = (
    "species", "l_max", "k_max", "body_order", "rb_size", "basics", "moments", "products",
    "scalars", "rows", "layers", "terminal_rows", "value_slots", "program_rows",
    "standard_graph_matched", "use_float", "neighbor_capacity", "neighbor_builds", "launches",
    "shared_xi", "product_slots_in_hbm", "cg_jit", "cg_jit_registers", "cg_jit_compile_ms",
    "basic_block", "force_block", "edge_jit", "edge_jit_basic_registers", "edge_jit_force_registers",
    "edge_jit_compile_ms", "gate_mode", "cg_kind", "cg_loaded_registers", "cg_local_bytes", "cg_build",
    "cg_from_disk_cache", "batch_fused", "batch_fused_registers", "batch_fused_shape", "batch_fused_tile",
    "batch_fused_compile_ms",
)


def is_sus2_sh_potential_file(path: str) -> bool:
    """is_sus2_sh_potential_file (src/force/sus2_sh.cu:7771-7780)."""
    return bool(_lib.load().sus2sh_is_sus2_sh_file(path.encode()))


class Box:
    """GPUMD's Box as the engine needs it: ``cpu_h`` (columns a, b, c) and pbc."""

    def __init__(self, h, pbc=(1, 1, 1)):
        self.cpu_h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(9))
        self.pbc = np.ascontiguousarray(np.asarray(pbc, dtype=np.int32).reshape(3))

    @classmethod
    def orthorhombic(cls, lx, ly, lz, pbc=(1, 1, 1)):
        return cls([lx, 0, 0, 0, ly, 0, 0, 0, lz], pbc)

    def lengths(self):
        h = self.cpu_h.reshape(3, 3)
        return np.linalg.norm(h, axis=0)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream_ptr(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


class SUS2_SH:
    """SUS2_SH(file_potential, num_atoms, options) -> engine handle."""

    def __init__(self, file_potential: str, num_atoms: int = 0, options=()):
        lib = _lib.load()
        self._lib = lib
        opts = [o.encode() for o in options]
        arr = (ctypes.c_char_p * max(1, len(opts)))(*opts) if opts else None
        h = ctypes.c_void_p()
        _lib.check(lib.sus2sh_create(file_potential.encode(), int(num_atoms), len(opts),
                                     ctypes.cast(arr, ctypes.c_void_p) if arr else None,
                                     ctypes.byref(h)), "sus2sh_create")
        self._h = h
        self.rc = lib.sus2sh_cutoff(h)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sus2sh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        out = (ctypes.c_int * len(MODEL_INFO_FIELDS))()
        n = self._lib.sus2sh_model_info(self._h, out, len(MODEL_INFO_FIELDS))
        return {k: out[i] for i, k in enumerate(MODEL_INFO_FIELDS[:n])}

    # --- GPUMD Potential::compute -----------------------------------------
    def compute(self, box: Box, type_, position, potential, force, virial, stream=None):
        """Accumulates E_i, F and W (all device tensors, GPUMD layouts)."""
        N = type_.numel()
        _lib.check(self._lib.sus2sh_compute(
            self._h, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p), box.pbc.ctypes.data_as(ctypes.c_void_p),
            _ptr(type_), _ptr(position), _ptr(potential), _ptr(force), _ptr(virial),
            _stream_ptr(stream)), "sus2sh_compute")

    def forward(self, box: Box, type_, position, potential, stream=None):
        N = type_.numel()
        _lib.check(self._lib.sus2sh_forward(
            self._h, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p), box.pbc.ctypes.data_as(ctypes.c_void_p),
            _ptr(type_), _ptr(position), _ptr(potential), _stream_ptr(stream)), "sus2sh_forward")

    def backward(self, grad_potential, grad_position, virial=None, stream=None):
        _lib.check(self._lib.sus2sh_backward(self._h, _ptr(grad_potential), _ptr(grad_position),
                                             _ptr(virial), _stream_ptr(stream)), "sus2sh_backward")

    def compute_host(self, box: Box, type_np, position_np, stream=None):
        """Host arrays in, (pe[N], force[3,N], virial_total[9]) out."""
        N = type_np.shape[0]
        t = np.ascontiguousarray(type_np, dtype=np.int32)
        p = np.ascontiguousarray(position_np, dtype=np.float64)
        pe = np.zeros(N)
        f = np.zeros((3, N))
        vt = np.zeros(9)
        s = _stream_ptr(stream) if stream is not None else None
        _lib.check(self._lib.sus2sh_compute_host(
            self._h, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p), box.pbc.ctypes.data_as(ctypes.c_void_p),
            t.ctypes.data_as(ctypes.c_void_p), p.ctypes.data_as(ctypes.c_void_p),
            pe.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
            vt.ctypes.data_as(ctypes.c_void_p), s), "sus2sh_compute_host")
        return pe, f, vt

    def compute_host_ptrs(self, box: Box, N, type_ptr, pos_ptr, pe_ptr, f_ptr, vt_ptr, stream=None):
        """Same as compute_host with raw (pinned) host pointers."""
        _lib.check(self._lib.sus2sh_compute_host(
            self._h, N, box.cpu_h.ctypes.data_as(ctypes.c_void_p), box.pbc.ctypes.data_as(ctypes.c_void_p),
            ctypes.c_void_p(type_ptr), ctypes.c_void_p(pos_ptr), ctypes.c_void_p(pe_ptr),
            ctypes.c_void_p(f_ptr), ctypes.c_void_p(vt_ptr), _stream_ptr(stream)), "sus2sh_compute_host")

    def compute_batch(self, cell_offset, cell_h, type_, position, potential, force, virial, cell_pbc=None,
                      cell_energy=None, cell_virial=None, stream=None):
        """Batch of independent cells (device tensors; see sus2sh_compute_batch)."""
        N = type_.numel()
        ncells = cell_offset.numel() - 1
        _lib.check(self._lib.sus2sh_compute_batch(
            self._h, N, ncells, _ptr(cell_offset), _ptr(cell_h), _ptr(cell_pbc), _ptr(type_), _ptr(position),
            _ptr(potential), _ptr(force), _ptr(virial), _ptr(cell_energy), _ptr(cell_virial),
            _stream_ptr(stream)), "sus2sh_compute_batch")

    def param_grad_batch(self, cell_offset, cell_h, type_, position, energy_weight, force_weight, grad_w, grad_c,
                         cell_pbc=None, stream=None):
        N = type_.numel()
        ncells = cell_offset.numel() - 1
        _lib.check(self._lib.sus2sh_param_grad_batch(
            self._h, N, ncells, _ptr(cell_offset), _ptr(cell_h), _ptr(cell_pbc), _ptr(type_), _ptr(position),
            _ptr(energy_weight), _ptr(force_weight), _ptr(grad_w), _ptr(grad_c), _stream_ptr(stream)),
            "sus2sh_param_grad_batch")

    def profile(self, enable: bool = True):
        _lib.check(self._lib.sus2sh_profile(self._h, 1 if enable else 0), "sus2sh_profile")

    def profile_read(self) -> dict:
        out = (ctypes.c_double * 6)()
        _lib.check(self._lib.sus2sh_profile_read(self._h, out, 6), "sus2sh_profile_read")
        keys = ("neighbor_ms", "basic_ms", "product_ms", "force_ms", "accumulate_ms", "calls")
        return {k: out[i] for i, k in enumerate(keys)}

    def sync(self) -> int:
        flags = ctypes.c_int(0)
        rc = self._lib.sus2sh_sync(self._h, ctypes.byref(flags))
        if rc not in (0, -4):
            _lib.check(rc, "sus2sh_sync")
        return flags.value


def standard_graph_counts(l_max, k_max, body_order, body_l_max=None) -> dict:
    """Counts of the standard graph (libsus2sh_tools.so)."""
    lib = _lib.load_tools()
    out = (ctypes.c_int * 8)()
    bl = (ctypes.c_int * len(body_l_max))(*body_l_max) if body_l_max else None
    _lib.check_tools(lib.sus2sh_standard_graph_counts(l_max, k_max, body_order,
                                                ctypes.cast(bl, ctypes.c_void_p) if bl else None,
                                                len(body_l_max) if body_l_max else 0, out),
               "sus2sh_standard_graph_counts")
    keys = ("node_count", "basics", "products", "scalars", "tensor_blocks", "cg_blocks", "cg_terms", "max_layer")
    return {k: out[i] for i, k in enumerate(keys)}
