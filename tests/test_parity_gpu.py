"""Parity of the CUDA engine (through the C-ABI) with the FP64 oracle.

Bars: FP32 engine within 1e-6 eV/atom energy and
1e-5 eV/A force RMS of the FP64 oracle; the FP64 engine within 1e-9.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, Box, structures  # noqa: E402

E_TOL32 = 1e-6      # eV/atom (or relative, see compare)
F_RMS32 = 1e-5      # eV/A
W_RMS32 = 1e-5      # eV per atom virial component
TOL64 = 1e-9


def engine_efs(path, box, types, pos, opts=(), species=("Cu", "Zr")):
    N = types.size
    pot = SUS2_SH(path, N, [*species, *opts])
    dev = torch.device("cuda")
    t = torch.as_tensor(types.astype(np.int32), device=dev)
    x = torch.as_tensor(np.ascontiguousarray(pos).reshape(-1), device=dev)
    pe = torch.zeros(N, dtype=torch.float64, device=dev)
    f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
    pot.compute(box, t, x, pe, f, w)
    torch.cuda.synchronize()
    assert pot.sync() == 0
    out = pe.cpu().numpy(), f.cpu().numpy().reshape(3, N), w.cpu().numpy().reshape(9, N)
    pot.close()
    return out


def compare(path, box, types, pos, opts=(), species=("Cu", "Zr"), fp64=False, relative=False):
    """relative=True divides the errors by the oracle's energy / force / virial
    scale (for synthetic models whose energies are far from physical)."""
    orc = O.Oracle(path)
    pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types, pos)
    pe, f, w = engine_efs(path, box, types, pos, opts=opts + (("sus2_float=0",) if fp64 else ()),
                          species=species)
    de = np.abs(pe - pe0).max()
    frms = np.sqrt(((f - f0) ** 2).mean())
    wrms = np.sqrt(((w - w0) ** 2).mean())
    if relative:
        # relative bars: energy 5e-6 of the largest site energy (FP32 moments
        # through a 33k-product graph), forces/virial 1e-5 of their RMS
        de = de / max(1.0, np.abs(pe0).max()) / 5.0
        frms /= max(1.0, np.sqrt((f0 ** 2).mean()))
        wrms /= max(1.0, np.sqrt((w0 ** 2).mean()))
    if fp64:
        assert de < TOL64 and np.abs(f - f0).max() < TOL64 * 10 and np.abs(w - w0).max() < TOL64 * 100, (de, frms, wrms)
    else:
        assert de < E_TOL32, de
        assert frms < F_RMS32, frms
        assert wrms < W_RMS32, wrms
    return de, frms, wrms


@pytest.mark.parametrize("fp64", [False, True])
def test_config0_fcc_2048(l3k3_path, fp64):
    box, types, pos = structures.fcc(8, 8, 8, 3.8, (0.5, 0.5), 0.05, seed=1)
    compare(l3k3_path, box, types, pos, fp64=fp64)


@pytest.mark.parametrize("fp64", [False, True])
def test_config0_row_interpreter(l3k3_path, fp64):
    # the generic CG row interpreter (used for large graphs) on the same case
    box, types, pos = structures.fcc(8, 8, 8, 3.8, (0.5, 0.5), 0.05, seed=1)
    compare(l3k3_path, box, types, pos, opts=("sus2_sh_cg_jit=0",), fp64=fp64)


@pytest.mark.parametrize("fp64", [False, True])
def test_small_periodic_cell_images(l3k3_path, fp64):
    # 3x3x3 FCC (11.4 A < 2 (rc + skin)): every neighbour image is explicit
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=2)
    compare(l3k3_path, box, types, pos, fp64=fp64)


def test_tiny_random_cell(l3k3_path):
    # 16 atoms at 0.06 A^-3 (edge about 6.4 A): images up to two boxes away
    box, types, pos = structures.random_insertion(16, 0.06, 2.1, (0.8, 1.0, 1.25), seed=3)
    compare(l3k3_path, box, types, pos)
    compare(l3k3_path, box, types, pos, fp64=True)


def test_triclinic_box(l3k3_path):
    box, types, pos = structures.fcc(5, 5, 5, 3.8, (0.5, 0.5), 0.05, seed=4)
    L = 19.0
    h = np.array([[L, 1.7, -0.9], [0.0, L, 2.3], [0.0, 0.0, L]])
    frac = np.linalg.solve(box.cpu_h.reshape(3, 3), pos)
    tbox = Box(h.ravel())
    compare(l3k3_path, tbox, types, h @ frac)


def test_open_boundaries(l3k3_path):
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=5)
    obox = Box.orthorhombic(60.0, 60.0, 60.0, pbc=(0, 0, 0))
    compare(l3k3_path, obox, types, pos + 20.0)
    mixed = Box.orthorhombic(11.4, 60.0, 11.4, pbc=(1, 0, 1))
    compare(l3k3_path, mixed, types, pos + np.array([[0.0], [20.0], [0.0]]))


def test_atoms_far_outside_an_open_axis(l3k3_path):
    # periodic x, y and open z with the box only 20 A high: clusters of the
    # crystal sit up to 150 A below and above it, where the neighbour fill's
    # cell-relative FP32 coordinates are large (tens of A) or beyond its FP32
    # limit (FP64 test for every candidate); the list must be the FP64 one
    box, types, pos = structures.fcc(3, 3, 2, 3.8, (0.5, 0.5), 0.05, seed=22)
    n = types.size
    shifts = np.array([-150.0, -60.0, 0.0, 45.0, 140.0])
    pos_all = np.concatenate([pos + np.array([[0.0], [0.0], [dz]]) for dz in shifts], axis=1)
    types_all = np.concatenate([types] * len(shifts))
    obox = Box.orthorhombic(11.4, 11.4, 20.0, pbc=(1, 1, 0))
    assert pos_all.shape[1] == n * len(shifts)
    compare(l3k3_path, obox, types_all, pos_all)
    compare(l3k3_path, obox, types_all, pos_all, fp64=True)


def test_dense_packing_overflows_the_fill_queue(l3k3_path):
    # 0.15 atoms/A^3 (about 136 neighbours within rc + skin): a neighbour cell
    # holds more candidates within the cutoff than the fill's per-thread queue,
    # so the fill takes its direct pass there; the list must stay the FP64 one
    box, types, pos = structures.random_insertion(900, 0.15, 1.6, (1.0, 1.1, 0.9), seed=23)
    compare(l3k3_path, box, types, pos, relative=True)
    compare(l3k3_path, box, types, pos, fp64=True, relative=True)


def per_mu_radial_model(src, dst):
    """Copy of model ``src`` whose radial functions each get their own (scal,
    shift) per species pair, so no radial argument is shared between them
    (scal_coeffs holds, per radial function, S*S scales then S*S shifts)."""
    import re
    text = open(src).read()
    S = int(re.search(r"species_count = (\d+)", text).group(1))
    m = re.search(r"scal_coeffs = \{([^}]*)\}", text)
    n = len(m.group(1).split(","))
    vals = []
    for mu in range(n // (2 * S * S)):
        vals += [0.8 + 0.07 * mu + 0.1 * p for p in range(S * S)]
        vals += [2.9 + 0.11 * mu - 0.05 * p for p in range(S * S)]
    text = text[:m.start(1)] + ", ".join(repr(v) for v in vals) + text[m.end(1):]
    with open(dst, "w") as fh:
        fh.write(text)
    return dst


def test_per_function_radial_arguments(l3k3_path, tmp_path):
    # every radial function with its own (scal, shift): the per-function
    # radial map of the moment and force kernels (the preset models share one
    # radial argument between all functions of a pair)
    path = per_mu_radial_model(l3k3_path, str(tmp_path / "per_mu.mtp"))
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.6, 0.4), 0.08, seed=21)
    pe0, f0, w0 = O.Oracle(path).efs(box.cpu_h, box.pbc, types, pos)
    pe, f, w = engine_efs(path, box, types, pos)
    # this model's site energies are larger than the preset's; single FP32
    # site energies reach about 1.4e-6 eV, so, as for the hot MD frame, the
    # energy bar is per atom of the system, with an RMS and a 5x max bar per site
    de = pe - pe0
    assert abs(de.sum()) / de.size < E_TOL32, de.sum()
    assert np.sqrt((de ** 2).mean()) < E_TOL32, np.sqrt((de ** 2).mean())
    assert np.abs(de).max() < 5 * E_TOL32, np.abs(de).max()
    assert np.sqrt(((f - f0) ** 2).mean()) < F_RMS32
    assert np.sqrt(((w - w0) ** 2).mean()) < W_RMS32
    compare(path, box, types, pos, fp64=True)


@pytest.mark.parametrize("opts", [(), ("sus2_sh_cg_split=0",)], ids=["split_kernel", "row_interpreter"])
def test_large_model_rational_three_species(l4k4_path, opts):
    # body-5 L=4 K=4 graph: the component-split CG kernel (default for this
    # size) and the row interpreter (product slots in HBM scratch).  The random
    # model has site energies up to ~5e2 eV and force RMS ~4e2 eV/A, so the FP32
    # bars are relative: 1e-6 of the energy scale, 1e-5 of the force / virial RMS.
    box, types, pos = structures.random_insertion(600, 0.06, 2.1, (1.0, 1.0, 1.0), (0.5, 0.35, 0.15), seed=6)
    compare(l4k4_path, box, types, pos, opts=opts, species=("Cu", "Zr", "Al"), relative=True)
    compare(l4k4_path, box, types, pos, opts=opts, species=("Cu", "Zr", "Al"), fp64=True, relative=True)


def test_large_model_uses_split_kernel(l4k4_path):
    box, types, pos = structures.random_insertion(300, 0.06, 2.1, (1.0, 1.0, 1.0), (0.5, 0.35, 0.15), seed=8)
    pot = SUS2_SH(l4k4_path, types.size, ["Cu", "Zr", "Al"])
    dev = torch.device("cuda")
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)
    pot.compute(box, torch.as_tensor(types, device=dev), torch.as_tensor(pos.reshape(-1).copy(), device=dev),
                z(types.size), z(3 * types.size), z(9 * types.size))
    torch.cuda.synchronize()
    info = pot.info()
    pot.close()
    assert info["cg_kind"] == 2 and 0 < info["cg_loaded_registers"] <= 255
    assert info["cg_build"] == 1  # one program (the default)
    assert info["cg_local_bytes"] <= 1024, info["cg_local_bytes"]


@pytest.mark.parametrize("fp64", [False, True])
def test_split_kernel_builds_agree_bit_for_bit(l4k4_path, fp64):
    # the one-program build (default) and the parallel relocatable build
    # (sus2_sh_cg_whole=0) compile the same source: identical site energies
    # and per-atom virials (each a per-centre sum of the CG kernel's outputs);
    # the forces are scattered with FP32 atomics, whose order varies from run
    # to run, so they agree to FP32 rounding
    box, types, pos = structures.random_insertion(2000, 0.06, 2.1, (1.0, 1.0, 1.0), (0.5, 0.35, 0.15), seed=9)
    base = ("sus2_float=0",) if fp64 else ()
    out = []
    for opts in (base, base + ("sus2_sh_cg_whole=0",)):
        out.append(engine_efs(l4k4_path, box, types, pos, opts, species=("Cu", "Zr", "Al")))
        pot = SUS2_SH(l4k4_path, types.size, ["Cu", "Zr", "Al", *opts])
        info = pot.info()
        pot.close()
        assert info["cg_kind"] == 2 and info["cg_build"] == (2 if "sus2_sh_cg_whole=0" in opts else 1), info
    (pe0, f0, w0), (pe1, f1, w1) = out
    assert np.array_equal(pe0, pe1) and np.array_equal(w0, w1)
    assert np.abs(f0 - f1).max() <= 1e-6 * np.abs(f0).max()


@pytest.mark.parametrize("fp64", [False, True])
def test_config0_split_kernel(l3k3_path, fp64):
    # the component-split CG kernel forced on the l3k3 model (120 one-value components)
    box, types, pos = structures.fcc(8, 8, 8, 3.8, (0.5, 0.5), 0.05, seed=1)
    compare(l3k3_path, box, types, pos, opts=("sus2_sh_cg_split=1",), fp64=fp64)


def test_reference_rounding_option(l3k3_path):
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.05, seed=7)
    orc = O.Oracle(l3k3_path, reference_rounding=True)
    pe0, f0, _ = orc.efs(box.cpu_h, box.pbc, types, pos)
    pe, f, _ = engine_efs(l3k3_path, box, types, pos, opts=("sus2_float=0", "sus2_sh_reference_rounding=1"))
    assert np.abs(pe - pe0).max() < 1e-9 and np.abs(f - f0).max() < 1e-8


def test_accumulates_into_outputs(l3k3_path):
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.05, seed=8)
    N = types.size
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"])
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    pe = torch.full((N,), 1.5, dtype=torch.float64, device=dev)
    f = torch.full((3 * N,), -0.25, dtype=torch.float64, device=dev)
    w = torch.full((9 * N,), 2.0, dtype=torch.float64, device=dev)
    pot.compute(box, t, x, pe, f, w)
    torch.cuda.synchronize()
    pe1, f1, w1 = engine_efs(l3k3_path, box, types, pos)
    # energies and virials are summed per centre atom (deterministic); forces
    # also receive FP32 atomics whose order varies between runs
    assert np.allclose(pe.cpu().numpy() - 1.5, pe1, atol=1e-12)
    assert np.allclose(f.cpu().numpy() + 0.25, f1.ravel(), atol=1e-6)
    assert np.allclose(w.cpu().numpy() - 2.0, w1.ravel(), atol=1e-12)


def test_deterministic_energy(l3k3_path):
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.5, 0.5), 0.05, seed=9)
    a = engine_efs(l3k3_path, box, types, pos)
    b = engine_efs(l3k3_path, box, types, pos)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[2], b[2])
    assert np.abs(a[1] - b[1]).max() < 1e-6


def test_md_steps_with_skin_rebuilds(l3k3_path):
    from sus2sh.md import NVE
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.64, 0.36), 0.05, seed=10)
    masses = [structures.AMU["Cu"], structures.AMU["Zr"]]
    vel = structures.maxwell_boltzmann(types, masses, 2000.0, seed=11)  # hot: forces rebuilds
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr", "sus2_sh_rebuild_interval=10"])
    md = NVE(pot, box, types, pos, vel, masses, dt_fs=2.0)
    md.initial_force()
    for _ in range(40):
        md.step()
    torch.cuda.synchronize()
    assert pot.sync() == 0
    assert pot.info()["neighbor_builds"] >= 4
    # the engine's forces at the final positions match the oracle there
    xf = md.pos.view(3, -1).cpu().numpy()
    orc = O.Oracle(l3k3_path)
    pe0, f0, _ = orc.efs(box.cpu_h, box.pbc, types, xf)
    pe = md.pe.cpu().numpy()
    # energy per atom (system energy / N) within the 1e-6 eV/atom bar; on this
    # hot (2000 K) frame single FP32 site energies reach about 1e-6 eV (RMS
    # about 1.3e-7), so the per-site errors get an RMS bar and a 5x max bar
    assert abs(pe.sum() - pe0.sum()) / pe.size < E_TOL32
    assert np.sqrt(((pe - pe0) ** 2).mean()) < E_TOL32
    assert np.abs(pe - pe0).max() < 5 * E_TOL32
    assert np.sqrt(((md.force.view(3, -1).cpu().numpy() - f0) ** 2).mean()) < F_RMS32


def test_neighbor_graph_matches_plain_launches(l3k3_path):
    # the neighbour work after the rebuild decision as a CUDA graph with IF
    # nodes (skipping the rebuild kernels on steps without a build) against
    # the plain launches: the same energies for the same positions (bit for
    # bit: no atomics in the energy), the same builds over a hot MD run, and the
    # same end of the run within FP32 rounding (the F_j scatter's FP32 atomics
    # add in a varying order, so two runs drift apart at the 1e-8 eV level)
    from sus2sh.md import NVE
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.64, 0.36), 0.05, seed=10)
    masses = [structures.AMU["Cu"], structures.AMU["Zr"]]
    vel = structures.maxwell_boltzmann(types, masses, 2000.0, seed=11)
    out = []
    for graph in (1, 0):
        pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr", "sus2_sh_rebuild_interval=7",
                                              f"sus2_sh_neighbor_graph={graph}"])
        md = NVE(pot, box, types, pos, vel, masses, dt_fs=2.0)
        md.initial_force()
        torch.cuda.synchronize()
        pe0 = md.pe.cpu().numpy().copy()
        for _ in range(30):
            md.step()
        torch.cuda.synchronize()
        assert pot.sync() == 0
        out.append((pe0, md.pe.cpu().numpy().copy(), md.force.cpu().numpy().copy(), pot.info()["neighbor_builds"]))
        pot.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][3] == out[1][3] >= 4
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-6
    assert np.sqrt(((out[0][2] - out[1][2]) ** 2).mean()) < 1e-5


def test_neighbor_overflow_is_reported_and_recovered(l3k3_path):
    # dilute first frame sizes the list; a compressed cluster then overflows it
    rng = np.random.default_rng(12)
    N = 200
    box = Box.orthorhombic(40.0, 40.0, 40.0)
    pos = rng.uniform(0, 40.0, size=(3, N))
    types = rng.integers(0, 2, N).astype(np.int32)
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"])
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)
    pot.compute(box, t, torch.as_tensor(pos.reshape(-1).copy(), device=dev), z(N), z(3 * N), z(9 * N))
    torch.cuda.synchronize()
    assert pot.sync() == 0
    dense = 15.0 + rng.uniform(0, 9.0, size=(3, N))  # ~0.27 A^-3 cluster
    x = torch.as_tensor(dense.reshape(-1).copy(), device=dev)
    pot.compute(box, t, x, z(N), z(3 * N), z(9 * N))
    assert pot.sync() & 1  # overflow flagged, capacity grown
    pe, f, w = z(N), z(3 * N), z(9 * N)
    pot.compute(box, t, x, pe, f, w)
    assert pot.sync() == 0
    orc = O.Oracle(l3k3_path)
    pe0, f0, _ = orc.efs(box.cpu_h, box.pbc, types, dense)
    assert np.abs(pe.cpu().numpy() - pe0).max() < 1e-4 * max(1.0, np.abs(pe0).max())


def test_autograd_backward_matches_forces_and_fd(l3k3_path):
    from sus2sh.autograd import site_energy
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=13)
    N = types.size
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    orc = O.Oracle(l3k3_path)
    pe0, f0, _ = orc.efs(box.cpu_h, box.pbc, types, pos)
    for fp64 in (False, True):
        pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
        x = torch.as_tensor(pos.reshape(-1).copy(), device=dev).requires_grad_(True)
        e = site_energy(pot, box, t, x)
        (g,) = torch.autograd.grad(e.sum(), x)
        assert np.abs(e.detach().cpu().numpy() - pe0).max() < (1e-10 if fp64 else E_TOL32)
        assert np.abs(g.cpu().numpy().reshape(3, N) + f0).max() < (1e-9 if fp64 else 1e-4)
        # weighted energies: gradient vs central differences of the oracle
        wts = np.random.default_rng(14).normal(size=N)
        e = site_energy(pot, box, t, x)
        (g,) = torch.autograd.grad((e * torch.as_tensor(wts, device=dev)).sum(), x)
        g = g.cpu().numpy().reshape(3, N)
        h = 1e-5
        for i in (0, 7, 33):
            for a in range(3):
                p1 = pos.copy(); p1[a, i] += h
                p2 = pos.copy(); p2[a, i] -= h
                fd = (wts @ orc.efs(box.cpu_h, box.pbc, types, p1)[0]
                      - wts @ orc.efs(box.cpu_h, box.pbc, types, p2)[0]) / (2 * h)
                assert abs(fd - g[a, i]) < (1e-7 if fp64 else 1e-4)
        pot.close()


def test_host_buffer_entry_point(l3k3_path):
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.05, seed=15)
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"])
    pe, f, vt = pot.compute_host(box, types, pos)
    orc = O.Oracle(l3k3_path)
    pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types, pos)
    assert np.abs(pe - pe0).max() < E_TOL32
    assert np.sqrt(((f - f0) ** 2).mean()) < F_RMS32
    assert np.abs(vt - w0.sum(axis=1)).max() < 1e-3
