"""Seeded synthetic SUS2-SH models of the benchmark workloads.

The reference's trained Cu-Zr models are not shipped, so every workload uses a
model written by ``sus2sh_write_synthetic_model`` (libsus2sh_tools.so:
standard real-CG graph, random coefficients).  Choices not fixed by the workload description are
recorded here: species_coeffs = 1, radial type coefficients = 1, every radial
(scal, shift) = (1.0, (r_min + rc)/2), and the Al site shift -3.0 eV.
"""
from __future__ import annotations

import ctypes
import os

from . import _lib

# name -> writer arguments
PRESETS = {
    # l3k3 Cu-Zr body-4 model: L=3, K=3, Chebyshev-sss rb=8, r_min 2.0, rc 5.0
    "l3k3": dict(species=2, l_max=3, k_max=3, body_order=4, rb_size=8, r_min=2.0, rc=5.0,
                 rational=0, shift=(-3.5, -5.0), radial_sigma=0.1, moment_sigma=0.01, seed=20260101),
    # second seeded model of the same shape (targets of the loss workload)
    "l3k3_target": dict(species=2, l_max=3, k_max=3, body_order=4, rb_size=8, r_min=2.0, rc=5.0,
                        rational=0, shift=(-3.5, -5.0), radial_sigma=0.1, moment_sigma=0.01, seed=20260202),
    # Cu-Zr-Al body-5 model: L=4, K=4, Chebyshev-sss-rational rb=10, rc 6.0
    "l4k4": dict(species=3, l_max=4, k_max=4, body_order=5, rb_size=10, r_min=2.0, rc=6.0,
                 rational=1, shift=(-3.5, -5.0, -3.0), radial_sigma=0.1, moment_sigma=0.01, seed=20260303),
}


def write_model(path: str, species=2, l_max=3, k_max=3, body_order=4, rb_size=8, r_min=2.0, rc=5.0,
                rational=0, shift=(-3.5, -5.0), radial_sigma=0.1, moment_sigma=0.01, scal=1.0,
                rshift=-1.0, seed=0, body_l_max=None, laguerre=False) -> str:
    """rational: 0 Chebyshev-sss, 1 its rational map; laguerre=True writes the
    Laguerre-log1p basis (rshift is then rho)."""
    lib = _lib.load_tools()
    sh = (ctypes.c_double * species)(*shift)
    bl = (ctypes.c_int * len(body_l_max))(*body_l_max) if body_l_max else None
    _lib.check_tools(lib.sus2sh_write_synthetic_model(
        path.encode(), species, l_max, k_max, body_order, ctypes.cast(bl, ctypes.c_void_p) if bl else None,
        len(body_l_max) if body_l_max else 0, rb_size, r_min, rc, 2 if laguerre else rational,
        ctypes.cast(sh, ctypes.c_void_p), radial_sigma, moment_sigma, scal, rshift,
        ctypes.c_ulonglong(seed)), "sus2sh_write_synthetic_model")
    return path


def preset_model(name: str, directory: str) -> str:
    """Writes preset ``name`` into ``directory`` (once) and returns the path."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, f"{name}.mtp")
    if not os.path.exists(path):
        write_model(path + ".tmp", **PRESETS[name])
        os.replace(path + ".tmp", path)
    return path


def add_zbl(src: str, dst: str, atomic_numbers=None, inner=None, outer=None, typewise=None, factor=None,
            enabled: str = "1") -> str:
    """Copies model ``src`` to ``dst`` with ZBL metadata appended (the keys
    load_sh_model reads, src/force/sus2_sh.cu:2132-2147); None leaves a key
    out so the reader's default applies."""
    with open(src) as fh:
        text = fh.read()
    lines = [f"zbl_enabled = {enabled}"]
    if inner is not None:
        lines.append(f"zbl_inner = {inner!r}")
    if outer is not None:
        lines.append(f"zbl_outer = {outer!r}")
    if typewise is not None:
        lines.append(f"zbl_typewise_cutoff_enabled = {1 if typewise else 0}")
    if factor is not None:
        lines.append(f"zbl_typewise_cutoff_factor = {factor!r}")
    if atomic_numbers is not None:
        lines.append("zbl_atomic_numbers = {" + ", ".join(str(int(z)) for z in atomic_numbers) + "}")
    with open(dst + ".tmp", "w") as fh:
        fh.write(text.rstrip("\n") + "\n" + "\n".join(lines) + "\n")
    os.replace(dst + ".tmp", dst)
    return dst


def add_gate(src: str, dst: str, mode: str = "mu-scalar-full", seed: int = 0, amplitude: float = 0.5,
             radial_sigma: float = 0.1, weight_sigma: float = 0.002, mix_sigma: float = 1.0,
             additive=None) -> str:
    """Copies model ``src`` to ``dst`` as a two-layer mu-body gate model (keys of
    load_sh_model, src/force/sus2_sh.cu:2153-2268): every scalar whose body
    order is at most sh_k_max + 1 is a gate signal, gate radial coefficients
    ~N(0, radial_sigma), signal weights ~N(0, weight_sigma), body-mix weights
    ~N(0, mix_sigma) (mu-body-linear-combo), seeded."""
    import re

    import numpy as np

    with open(src) as fh:
        text = fh.read()

    def value(key):
        return re.search(re.escape(key) + r"\s*(\S+)", text).group(1)

    K = int(value("sh_k_max ="))
    L = int(value("sh_l_max ="))
    rb = int(value("radial_basis_size ="))
    S = int(value("species_count ="))
    kmu = K * (L + 1)
    info = re.search(r"sh_scalar_info = \{(.*)\}\s*$", text, re.M).group(1)
    bodies = [int(b) for b in re.findall(r"\{(\d+)", info)]
    qidx = [q for q, b in enumerate(bodies) if b <= K + 1]
    rng = np.random.default_rng(seed)
    fmt = lambda v: "{" + ", ".join(repr(float(x)) for x in v) + "}"  # noqa: E731
    lines = ["two_layer_gate_enabled = 1", f"two_layer_gate_mode = {mode}", "two_layer_gate_site_mode = neighbor",
             "two_layer_gate_radial_mode = shared-radial", f"two_layer_gate_tanh_amplitude = {amplitude!r}",
             f"two_layer_gate_body_order_max = {K + 1}",
             f"two_layer_gate_radial_coeff_count = {kmu * rb}",
             "two_layer_gate_radial_coeffs = " + fmt(rng.normal(0.0, radial_sigma, kmu * rb))]
    if additive is not None:
        lines += [f"two_layer_gate_additive_coeff_count = {S}", "two_layer_gate_additive_coeffs = " + fmt(additive)]
    nw = kmu * len(qidx) if mode != "mu-body-linear-combo" else len(qidx)
    lines += [f"two_layer_gate_weight_count = {nw}",
              "two_layer_gate_scalar_indices = {" + ", ".join(str(q) for q in qidx) + "}",
              "two_layer_gate_weights = " + fmt(rng.normal(0.0, weight_sigma, nw))]
    if mode == "mu-body-linear-combo":
        lines += [f"two_layer_gate_body_mix_weight_count = {kmu * K}",
                  "two_layer_gate_body_mix_weights = " + fmt(rng.normal(0.0, mix_sigma, kmu * K))]
    with open(dst + ".tmp", "w") as fh:
        fh.write(text.rstrip("\n") + "\n" + "\n".join(lines) + "\n")
    os.replace(dst + ".tmp", dst)
    return dst
