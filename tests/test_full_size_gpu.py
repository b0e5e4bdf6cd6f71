"""Parity at the workloads' real sizes, against the FP64 oracle.

* The 1,024,000-atom l3k3 Cu-Zr crystal (80 x 80 x 40 FCC, 64/36, a thermal
  frame: N(0, 0.03 A) displacements), FP32 engine: energy per atom within
  1e-6 eV, site energies RMS 1e-6 and at most 5e-6 eV, force and virial RMS
  1e-5 (the oracle takes a few seconds on the host cores).
* The 4,096-cell uneven batch of the benchmark (16-512 atoms per cell,
  1.08M atoms), FP32 engine, cell by cell: the same bars, per cell; and the
  batched parameter gradients of the FP32 engine against the FP64 engine's.
* The 262,144-atom Cu-Zr-Al l4k4 body-5 rational workload's model on 32,768
  atoms of the same density (the oracle's cost grows with the 33,389
  products per atom): absolute errors printed, bars relative to the site
  energies (up to ~5e2 eV on this random model): 5e-6 of the largest site
  energy, force and virial RMS 1e-5 of their RMS.
The parameter gradients on 64 cells of 108 atoms are in test_param_grad_gpu.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, structures  # noqa: E402
from test_parity_gpu import engine_efs  # noqa: E402


def _errors(pe, f, w, pe0, f0, w0):
    de = pe - pe0
    return {"dE_per_atom": abs(float(de.sum())) / de.size, "site_rms": float(np.sqrt((de ** 2).mean())),
            "site_max": float(np.abs(de).max()), "force_rms": float(np.sqrt(((f - f0) ** 2).mean())),
            "virial_rms": float(np.sqrt(((w - w0) ** 2).mean()))}


def test_million_atom_crystal_fp32_vs_oracle(l3k3_path):
    box, types, pos = structures.fcc(80, 80, 40, 3.8, (0.64, 0.36), 0.03, seed=1000)
    pe, f, w = engine_efs(l3k3_path, box, types, pos)
    pe0, f0, w0 = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, pos)
    e = _errors(pe, f, w, pe0, f0, w0)
    print("1.024M-atom l3k3 FP32 vs FP64 oracle:", e)
    assert e["dE_per_atom"] < 1e-6 and e["site_rms"] < 1e-6 and e["site_max"] < 5e-6, e
    assert e["force_rms"] < 1e-5 and e["virial_rms"] < 1e-5, e


def _batch_run(pot, off, H, types, pos):
    dev = torch.device("cuda")
    N = types.size
    T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a).reshape(-1), dtype=dt, device=dev)  # noqa: E731
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
    pe, f, w = z(N), z(3 * N), z(9 * N)
    pot.compute_batch(T(off, torch.int32), T(H), T(types, torch.int32), T(pos), pe, f, w)
    torch.cuda.synchronize()
    assert pot.sync() == 0
    return pe.cpu().numpy(), f.view(3, N).cpu().numpy(), w.view(9, N).cpu().numpy()


def test_4096_cell_batch_fp32_vs_oracle(l3k3_path):
    off, H, boxes, types, pos = structures.cell_batch(4096, 16, 512, seed=4242)  # the benchmark's batch
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"])
    pe, f, w = _batch_run(pot, off, H, types, pos)
    pot.close()
    orc = O.Oracle(l3k3_path)
    worst = {}
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        e = _errors(pe[a:b], f[:, a:b], w[:, a:b], pe0, f0, w0)
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
    print("4096-cell batch FP32 vs FP64 oracle, worst cell:", worst)
    assert worst["dE_per_atom"] < 1e-6 and worst["site_rms"] < 1e-6 and worst["site_max"] < 5e-6, worst
    assert worst["force_rms"] < 1e-5 and worst["virial_rms"] < 1e-5, worst


def test_4096_cell_batch_parameter_gradients_fp32_vs_fp64(l3k3_path):
    off, H, boxes, types, pos = structures.cell_batch(4096, 16, 512, seed=4242)
    N = types.size
    dev = torch.device("cuda")
    T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a).reshape(-1), dtype=dt, device=dev)  # noqa: E731
    rng = np.random.default_rng(3)
    ew = rng.normal(0.0, 1.0, N)
    fw = rng.normal(0.0, 0.1, (3, N))
    out = []
    for fp64 in (False, True):
        pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
        info = pot.info()
        nsc, nrad = info["scalars"], info["k_max"] * (info["l_max"] + 1) * info["rb_size"]
        gw = torch.zeros(nsc, dtype=torch.float64, device=dev)
        gc = torch.zeros(nrad, dtype=torch.float64, device=dev)
        pot.param_grad_batch(T(off, torch.int32), T(H), T(types, torch.int32), T(pos), T(ew), T(fw), gw, gc)
        torch.cuda.synchronize()
        assert pot.sync() == 0
        out.append((gw.cpu().numpy(), gc.cpu().numpy()))
        pot.close()
    (gw32, gc32), (gw64, gc64) = out
    rel_w = np.abs(gw32 - gw64).max() / np.abs(gw64).max()
    rel_c = np.abs(gc32 - gc64).max() / np.abs(gc64).max()
    print("4096-cell batched parameter gradients, FP32 vs FP64, largest error / largest gradient:",
          {"moment_coeffs": rel_w, "radial_coeffs": rel_c})
    assert rel_w < 1e-5 and rel_c < 1e-5, (rel_w, rel_c)


def test_large_model_absolute_errors(l4k4_path):
    box, types, pos = structures.random_insertion(32768, 0.06, 2.1, (1.0, 1.0, 1.0), (0.5, 0.35, 0.15), seed=77)
    pe0, f0, w0 = O.Oracle(l4k4_path).efs(box.cpu_h, box.pbc, types, pos)
    pe, f, w = engine_efs(l4k4_path, box, types, pos, (), species=("Cu", "Zr", "Al"))
    e = _errors(pe, f, w, pe0, f0, w0)
    scales = {"site_energy_max": float(np.abs(pe0).max()), "force_rms": float(np.sqrt((f0 ** 2).mean())),
              "virial_rms": float(np.sqrt((w0 ** 2).mean()))}
    print("l4k4 body-5 rational, 32,768 atoms, FP32 vs FP64 oracle (absolute):", e, "scales:", scales)
    assert e["site_max"] < 5e-6 * scales["site_energy_max"], (e, scales)
    assert e["force_rms"] < 1e-5 * scales["force_rms"] and e["virial_rms"] < 1e-5 * scales["virial_rms"], (e, scales)
