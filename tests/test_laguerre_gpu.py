"""The Laguerre-log1p radial basis (RBLaguerre_log1p, src/force/sus2_sh.cu:
363-374,3299-3352): phi_n(r) = (r - rc)^2 exp(-u/2) L_n(u), u = scal
log(1 + r / rho).

Parity of the engine with the FP64 oracle (every radial function of a pair on
one argument, and each with its own (scal, rho)), in the FP32 build
specialised to the model, the FP32 build reading the coefficients from its
parameters, and FP64; with the reference's own engine on the same inputs,
including the reference's smoke configuration (8 species, an H-C pair 2 A
apart in a 20 A box, codex_tests/laguerre_sh_gpumd_smoke_20260530); and the
parameter gradients against finite differences of the oracle's loss.
"""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import ref_engine  # noqa: E402
import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, Box, models, structures  # noqa: E402
from sus2sh.training import loss_and_grad  # noqa: E402
from test_parity_gpu import compare, engine_efs  # noqa: E402

E_TOL32, F_RMS32 = 1e-6, 1e-5


def _per_mu(src, dst):
    """Each radial function of each pair with its own (scal, rho)."""
    text = open(src).read()
    S = int(re.search(r"species_count = (\d+)", text).group(1))
    m = re.search(r"scal_coeffs = \{([^}]*)\}", text)
    n = len(m.group(1).split(","))
    vals = []
    for mu in range(n // (2 * S * S)):
        vals += [0.7 + 0.06 * mu + 0.1 * p for p in range(S * S)]
        vals += [1.5 + 0.2 * mu - 0.1 * p for p in range(S * S)]
    open(dst, "w").write(text[:m.start(1)] + ", ".join(repr(v) for v in vals) + text[m.end(1):])
    return dst


@pytest.mark.parametrize("opts", [(), ("sus2_sh_model_edges=0",)], ids=["model_build", "parameter_build"])
def test_crystal_and_small_cell(laguerre_path, opts):
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.5, 0.5), 0.05, seed=41)
    compare(laguerre_path, box, types, pos, opts=opts)
    box, types, pos = structures.fcc(2, 2, 1, 3.8, (0.5, 0.5), 0.08, seed=42)
    compare(laguerre_path, box, types, pos, opts=opts)
    compare(laguerre_path, box, types, pos, opts=opts, fp64=True)


def test_per_function_arguments(laguerre_path, tmp_path):
    path = _per_mu(laguerre_path, str(tmp_path / "lag_per_mu.mtp"))
    box, types, pos = structures.fcc(5, 5, 5, 3.8, (0.6, 0.4), 0.08, seed=43)
    compare(path, box, types, pos)
    compare(path, box, types, pos, fp64=True)


@pytest.mark.skipif(not ref_engine.available(), reason="oracle/_ref/ref_sus2sh not built")
def test_against_the_reference(laguerre_path, tmp_path):
    for path in (laguerre_path, _per_mu(laguerre_path, str(tmp_path / "lag_per_mu.mtp"))):
        box, types, pos = structures.fcc(5, 5, 5, 3.8, (0.5, 0.5), 0.05, seed=44)
        pe_r, f_r, w_r = ref_engine.run(path, box.cpu_h, box.pbc, types, pos, ("Cu", "Zr", "sus2_float=0"))[:3]
        fbar = 1e-6 * max(1.0, np.abs(f_r).max())
        pe, f, w = engine_efs(path, box, types, pos, ("sus2_float=0", "sus2_sh_reference_rounding=1"))
        assert np.abs(pe - pe_r).max() < 1e-9 and np.abs(f - f_r).max() < fbar
        pe, f, w = engine_efs(path, box, types, pos)
        assert np.abs(pe - pe_r).max() < E_TOL32 and np.sqrt(((f - f_r) ** 2).mean()) < F_RMS32
        pe_r32, f_r32 = ref_engine.run(path, box.cpu_h, box.pbc, types, pos, ("Cu", "Zr"))[:2]
        assert np.abs(pe - pe_r32).max() < 1e-5 and np.sqrt(((f - f_r32) ** 2).mean()) < 1e-4


@pytest.mark.skipif(not ref_engine.available(), reason="oracle/_ref/ref_sus2sh not built")
def test_reference_smoke_configuration(tmp_path):
    # 8 species (H C N O Cl K Co Ni), one H-C pair 2 A apart in a 20 A box
    syms = ("H", "C", "N", "O", "Cl", "K", "Co", "Ni")
    path = models.write_model(str(tmp_path / "lag8.mtp"), species=8, shift=tuple(-1.0 - 0.5 * s for s in range(8)),
                              laguerre=True, rb_size=10, rshift=1.0, seed=530)
    box = Box.orthorhombic(20.0, 20.0, 20.0)
    types = np.array([0, 1], dtype=np.int32)
    pos = np.array([[5.0, 7.0], [5.0, 5.0], [5.0, 5.0]])
    pe_r, f_r, w_r = ref_engine.run(path, box.cpu_h, box.pbc, types, pos, (*syms, "sus2_float=0"))[:3]
    pe0, f0, w0 = O.Oracle(path).efs(box.cpu_h, box.pbc, types, pos)
    pe, f, w = engine_efs(path, box, types, pos, ("sus2_float=0",), species=syms)
    assert np.abs(pe - pe0).max() < 1e-9 and np.abs(f - f0).max() < 1e-9
    assert np.abs(pe_r - pe0).max() < 1e-6 and np.abs(f_r - f0).max() < 1e-6 * max(1.0, np.abs(f0).max())
    pe, f, w = engine_efs(path, box, types, pos, (), species=syms)
    assert np.abs(pe - pe0).max() < E_TOL32 and np.abs(f - f0).max() < F_RMS32


@pytest.mark.parametrize("fp64", [True, False])
def test_param_grad_matches_finite_differences(laguerre_path, model_dir, fp64):
    tpath = models.write_model(f"{model_dir}/lag_target.mtp", laguerre=True, seed=20260405)
    cells = [structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=400 + c) for c in range(2)]
    torc = O.Oracle(tpath)
    targets = []
    for box, types, pos in cells:
        pe, f, _ = torc.efs(box.cpu_h, box.pbc, types, pos)
        targets.append((pe.sum(), f))
    pot = SUS2_SH(laguerre_path, cells[0][1].size, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    L, gw, gc = loss_and_grad(pot, cells, targets)
    pot.close()
    orc = O.Oracle(laguerre_path)

    def loss():
        out = 0.0
        for (box, types, pos), (Et, Ft) in zip(cells, targets):
            pe, f, _ = orc.efs(box.cpu_h, box.pbc, types, pos)
            out += (pe.sum() - Et) ** 2 + 0.1 * ((f - Ft) ** 2).sum()
        return out

    L0 = loss()
    assert abs(L - L0) < (1e-9 if fp64 else 1e-5) * max(1.0, abs(L0))
    rng = np.random.default_rng(7)
    h = 1e-4
    rel = 1e-5 if fp64 else 2e-3
    for g, arr, idxs in ((gw, orc.arrays.w, rng.choice(gw.size, 6, replace=False)),
                         (gc, orc.arrays.radial, rng.choice(gc.size, 8, replace=False))):
        scale = np.abs(g).max()
        for q in idxs:
            old = arr[q]
            arr[q] = old + h
            Lp = loss()
            arr[q] = old - h
            Lm = loss()
            arr[q] = old
            assert abs((Lp - Lm) / (2 * h) - g[q]) < rel * scale + 1e-7, (q, g[q])
