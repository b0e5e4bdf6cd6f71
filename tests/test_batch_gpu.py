"""Batches of small periodic cells of uneven size in one pass
(sus2sh_compute_batch / sus2sh_param_grad_batch), against the FP64 oracle
cell by cell, and captured in a CUDA graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, Box, structures  # noqa: E402


@pytest.fixture(scope="module")
def batch():
    return structures.cell_batch(24, 16, 512, seed=41)


def _run(pot, off, H, types, pos, dev, cell=True, pbc=None):
    N = types.size
    ncells = off.size - 1
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    o = torch.as_tensor(off, device=dev)
    h = torch.as_tensor(H.reshape(-1).copy(), device=dev)
    cp = torch.as_tensor(np.ascontiguousarray(pbc, dtype=np.int32).reshape(-1), device=dev) if pbc is not None else None
    pe = torch.zeros(N, dtype=torch.float64, device=dev)
    f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
    ce = torch.zeros(ncells, dtype=torch.float64, device=dev)
    cw = torch.zeros(9 * ncells, dtype=torch.float64, device=dev)
    pot.compute_batch(o, h, t, x, pe, f, w, cell_pbc=cp, cell_energy=ce, cell_virial=cw)
    torch.cuda.synchronize()
    assert pot.sync() == 0
    return pe.cpu().numpy(), f.view(3, N).cpu().numpy(), w.view(9, N).cpu().numpy(), ce.cpu().numpy(), \
        cw.view(ncells, 9).cpu().numpy()


@pytest.mark.parametrize("fp64", [False, True])
def test_batch_matches_oracle_cell_by_cell(l3k3_path, batch, fp64):
    off, H, boxes, types, pos = batch
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    pe, f, w, ce, cw = _run(pot, off, H, types, pos, dev)
    orc = O.Oracle(l3k3_path)
    etol, frms_tol = (1e-9, 1e-9) if fp64 else (1e-6, 1e-5)
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        assert np.abs(pe[a:b] - pe0).max() < etol
        assert np.sqrt(((f[:, a:b] - f0) ** 2).mean()) < frms_tol
        assert np.sqrt(((w[:, a:b] - w0) ** 2).mean()) < frms_tol
        assert abs(ce[c] - pe0.sum()) < etol * (b - a)
        assert np.abs(cw[c] - w0.sum(axis=1)).max() < frms_tol * (b - a)
    pot.close()


def test_batch_dense_wide_cells(l3k3_path):
    # cells wider than twice the cutoff: 256 atoms at 0.14 atoms/A^3 (one
    # tile, about 127 near candidates per atom) overflow the wide-cell path's
    # queue so its direct pass takes over; 700 atoms at 0.15 (three tiles) and
    # a cell of ordinary density stay within it
    cells = [structures.random_insertion(256, 0.14, 1.6, (1.0, 1.0, 1.0), seed=51),
             structures.random_insertion(300, 0.06, 2.1, (1.0, 1.0, 1.2), seed=52),
             structures.random_insertion(700, 0.15, 1.6, (1.1, 0.9, 1.0), seed=53)]
    boxes = [c[0] for c in cells]
    types = np.concatenate([c[1] for c in cells]).astype(np.int32)
    pos = np.concatenate([c[2] for c in cells], axis=1)
    off = np.concatenate([[0], np.cumsum([c[1].size for c in cells])]).astype(np.int32)
    H = np.stack([b.cpu_h.reshape(9) for b in boxes])
    assert all((np.diag(b.cpu_h.reshape(3, 3)) > 12.1).all() for b in boxes)
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"])
    pe, f, w, ce, cw = _run(pot, off, H, types, pos, dev)
    pot.close()
    orc = O.Oracle(l3k3_path)
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        # relative bars: dense random packings give large synthetic-model energies
        assert np.abs(pe[a:b] - pe0).max() < 5e-6 * max(1.0, np.abs(pe0).max())
        assert np.sqrt(((f[:, a:b] - f0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((f0 ** 2).mean()))
        assert np.sqrt(((w[:, a:b] - w0) ** 2).mean()) < 1e-5 * max(1.0, np.sqrt((w0 ** 2).mean()))


def _segments(nx, ny, nz, shifts, seed):
    """Copies of one FCC block shifted along z."""
    _, types, pos = structures.fcc(nx, ny, nz, 3.8, (0.5, 0.5), 0.05, seed=seed)
    return (np.concatenate([types] * len(shifts)).astype(np.int32),
            np.concatenate([pos + np.array([[0.0], [0.0], [s]]) for s in shifts], axis=1))


@pytest.mark.parametrize("fp64", [False, True])
def test_batch_cells_spread_over_thousands_of_angstrom(l3k3_path, fp64):
    # orthorhombic cells whose atoms lie thousands of A apart: a 7.6 x 7.6 x
    # 6000 A periodic wire of FCC segments (one across the z boundary) and a
    # cell periodic in x, y (15.2 A) with FCC slabs up to 7000 A out along
    # its open z axis.  Such cells take the FP64 image scan instead of the
    # FP32 pre-tests (whose margins hold for cell-local coordinates); a compact
    # cell after them keeps the shared-memory scan.  Lists and results must
    # be the oracle's.
    t1, p1 = _segments(2, 2, 3, [0.0, 1500.0, 3000.0, 5988.6], 61)
    p1[2] %= 6000.0
    t2, p2 = _segments(4, 4, 2, [0.0, -7000.0, -6992.4, 6000.0], 62)
    b3, t3, p3 = structures.fcc(4, 4, 4, 3.8, (0.64, 0.36), 0.05, seed=63)
    boxes = [Box.orthorhombic(7.6, 7.6, 6000.0), Box.orthorhombic(15.2, 15.2, 20.0, pbc=(1, 1, 0)), b3]
    types = np.concatenate([t1, t2, t3]).astype(np.int32)
    pos = np.concatenate([p1, p2, p3], axis=1)
    off = np.concatenate([[0], np.cumsum([t1.size, t2.size, t3.size])]).astype(np.int32)
    H = np.stack([b.cpu_h.reshape(9) for b in boxes])
    pbc = np.stack([b.pbc for b in boxes])
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else []))
    pe, f, w, ce, cw = _run(pot, off, H, types, pos, dev, pbc=pbc)
    pot.close()
    orc = O.Oracle(l3k3_path)
    etol, tol = (1e-9, 1e-9) if fp64 else (1e-6, 1e-5)
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        assert np.abs(pe[a:b] - pe0).max() < etol, c
        assert np.sqrt(((f[:, a:b] - f0) ** 2).mean()) < tol, c
        assert np.sqrt(((w[:, a:b] - w0) ** 2).mean()) < tol, c
        assert abs(ce[c] - pe0.sum()) < etol * (b - a), c


def test_batch_mixed_triclinic_cells(l3k3_path):
    # every other cell sheared (xy and xz tilts): triclinic cells take the
    # general per-atom image scan, orthorhombic ones the shared-memory scan
    off, H, boxes, types, pos = structures.cell_batch(8, 40, 300, seed=77)
    H = H.copy()
    pos = pos.copy()
    tboxes = []
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        h = box.cpu_h.reshape(3, 3).copy()
        if c % 2:
            frac = np.linalg.solve(h, pos[:, a:b])
            h[0, 1] = 0.12 * h[1, 1]
            h[0, 2] = -0.08 * h[2, 2]
            pos[:, a:b] = h @ frac
        H[c] = h.reshape(-1)
        tboxes.append(Box(h.reshape(-1), box.pbc))
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"])
    pe, f, w, ce, cw = _run(pot, off, H, types, pos, dev)
    orc = O.Oracle(l3k3_path)
    for c, box in enumerate(tboxes):
        a, b = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[a:b], pos[:, a:b])
        assert np.abs(pe[a:b] - pe0).max() < 1e-6, c
        assert np.sqrt(((f[:, a:b] - f0) ** 2).mean()) < 1e-5, c
        assert np.sqrt(((w[:, a:b] - w0) ** 2).mean()) < 1e-5, c
    pot.close()


def test_batch_in_a_cuda_graph(l3k3_path, batch):
    off, H, boxes, types, pos = batch
    dev = torch.device("cuda")
    N, ncells = types.size, off.size - 1
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"])
    ref = _run(pot, off, H, types, pos, dev)  # first call sizes the lists
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    o = torch.as_tensor(off, device=dev)
    h = torch.as_tensor(H.reshape(-1).copy(), device=dev)
    pe = torch.zeros(N, dtype=torch.float64, device=dev)
    f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
    w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
    ce = torch.zeros(ncells, dtype=torch.float64, device=dev)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        pe.zero_(); f.zero_(); w.zero_()
        pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce)  # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        pe.zero_(); f.zero_(); w.zero_()
        pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(pe.cpu().numpy(), ref[0])
    assert np.abs(f.view(3, N).cpu().numpy() - ref[1]).max() < 1e-6
    assert np.array_equal(ce.cpu().numpy(), ref[3])
    # new positions in the same buffers: the replay re-evaluates them
    pos2 = pos + np.random.default_rng(3).normal(0, 0.02, size=pos.shape)
    x.copy_(torch.as_tensor(pos2.reshape(-1)))
    g.replay()
    torch.cuda.synchronize()
    orc = O.Oracle(l3k3_path)
    for c in (0, 7, ncells - 1):
        a, b = off[c], off[c + 1]
        pe0, f0, _ = orc.efs(boxes[c].cpu_h, boxes[c].pbc, types[a:b], pos2[:, a:b])
        assert np.abs(pe.cpu().numpy()[a:b] - pe0).max() < 1e-6
    del g
    pot.close()


def test_param_grad_batch_equals_sum_over_cells(l3k3_path, batch):
    import ctypes
    off, H, boxes, types, pos = batch
    dev = torch.device("cuda")
    N = types.size
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr", "sus2_float=0"])
    info = pot.info()
    nsc, nrad = info["scalars"], info["k_max"] * (info["l_max"] + 1) * info["rb_size"]
    rng = np.random.default_rng(9)
    ew = rng.normal(size=N)
    fw = rng.normal(size=(3, N)) * 0.1
    T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    gw = torch.zeros(nsc, dtype=torch.float64, device=dev)
    gc = torch.zeros(nrad, dtype=torch.float64, device=dev)
    pot.param_grad_batch(T(off, torch.int32), T(H.reshape(-1)), T(types, torch.int32), T(pos.reshape(-1)),
                         T(ew), T(fw.reshape(-1)), gw, gc)
    torch.cuda.synchronize()
    from sus2sh import _lib
    lib = _lib.load()
    sw, sc = np.zeros(nsc), np.zeros(nrad)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    for c, box in enumerate(boxes):
        a, b = off[c], off[c + 1]
        n = b - a
        gw1 = torch.zeros(nsc, dtype=torch.float64, device=dev)
        gc1 = torch.zeros(nrad, dtype=torch.float64, device=dev)
        tt, xx = T(types[a:b], torch.int32), T(pos[:, a:b].reshape(-1))
        e1, f1 = T(ew[a:b]), T(fw[:, a:b].reshape(-1))
        rc = lib.sus2sh_param_grad(pot.handle, n, box.cpu_h.ctypes.data_as(ctypes.c_void_p),
                                   box.pbc.ctypes.data_as(ctypes.c_void_p), p(tt), p(xx), p(e1), p(f1),
                                   p(gw1), p(gc1), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        sw += gw1.cpu().numpy()
        sc += gc1.cpu().numpy()
    assert np.abs(gw.cpu().numpy() - sw).max() < 1e-9 * max(1.0, np.abs(sw).max())
    assert np.abs(gc.cpu().numpy() - sc).max() < 1e-9 * max(1.0, np.abs(sc).max())
    pot.close()


def _cells(specs, seed):
    """Concatenated random-insertion cells: specs = [(atoms, density, ratios)]."""
    cells = [structures.random_insertion(n, rho, 2.1, ratios, seed=seed + k) for k, (n, rho, ratios) in
             enumerate(specs)]
    boxes = [c[0] for c in cells]
    types = np.concatenate([c[1] for c in cells]).astype(np.int32)
    pos = np.concatenate([c[2] for c in cells], axis=1)
    off = np.concatenate([[0], np.cumsum([c[1].size for c in cells])]).astype(np.int32)
    H = np.stack([b.cpu_h.reshape(9) for b in boxes])
    return off, H, boxes, types, pos


@pytest.mark.parametrize("tile", [0, 256])
def test_fused_batch_kernel_matches_stage_kernels_and_oracle(l3k3_path, batch, tile):
    """The fused persistent batch kernel (sus2_sh_batch_fused=1) against the
    stage kernels (the default) on the same batch, and against
    the oracle cell by cell; tile 256 gives cells of up to 512 atoms
    several tiles' worth of atoms, so most tiles hold one or two cells."""
    off, H, boxes, types, pos = batch
    dev = torch.device("cuda")
    opts = ["Cu", "Zr", "sus2_sh_batch_fused=1"] + ([f"sus2_sh_batch_tile={tile}"] if tile else [])
    fused = SUS2_SH(l3k3_path, types.size, opts)
    stage = SUS2_SH(l3k3_path, types.size, ["Cu", "Zr"])
    a = _run(fused, off, H, types, pos, dev)
    b = _run(stage, off, H, types, pos, dev)
    info, info0 = fused.info(), stage.info()
    assert info["batch_fused"] == 1 and info0["batch_fused"] == 0
    if tile:
        assert info["batch_fused_tile"] == tile
    fused.close()
    stage.close()
    pe, f, w, ce, cw = a
    # same per-atom arithmetic; forces and virials differ by FP32 summation order
    assert np.abs(pe - b[0]).max() < 1e-9
    assert np.sqrt(((f - b[1]) ** 2).mean()) < 1e-6
    assert np.sqrt(((w - b[2]) ** 2).mean()) < 1e-6
    assert np.abs(ce - b[3]).max() < 1e-8
    assert np.abs(cw - b[4]).max() < 1e-5
    orc = O.Oracle(l3k3_path)
    for c, box in enumerate(boxes):
        lo, hi = off[c], off[c + 1]
        pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types[lo:hi], pos[:, lo:hi])
        assert np.abs(pe[lo:hi] - pe0).max() < 1e-6
        assert np.sqrt(((f[:, lo:hi] - f0) ** 2).mean()) < 1e-5
        assert np.sqrt(((w[:, lo:hi] - w0) ** 2).mean()) < 1e-5
        assert abs(ce[c] - pe0.sum()) < 1e-6 * (hi - lo)


def test_fused_batch_kernel_large_and_tiny_cells(l3k3_path):
    """Tiles whose atoms exceed the shared-memory force buffer (a 1,700-atom
    cell at tile 256: buffer of 1,536 atoms) take the FP64-atomic path; cells
    of one to three atoms (no neighbour within the cutoff) and an empty cell
    get their sums; outputs accumulate into non-zero arrays and the per-cell
    sums are assigned, as in the stage path; two calls in a row agree."""
    off, H, boxes, types, pos = _cells([(40, 0.06, (1.0, 1.0, 1.0)), (1700, 0.06, (1.0, 1.1, 0.9)),
                                        (300, 0.06, (1.2, 1.0, 1.0))], seed=71)
    # cells of 1, 3 and 0 atoms: 20 A cubes
    tiny = [np.zeros((3, 1)) + 3.0, np.array([[1.0, 8.0, 15.0], [2.0, 2.0, 9.0], [3.0, 14.0, 3.0]]),
            np.zeros((3, 0))]
    for p in tiny:
        boxes.append(Box.orthorhombic(20.0, 20.0, 20.0))
        H = np.vstack([H, boxes[-1].cpu_h.reshape(1, 9)])
        types = np.concatenate([types, np.arange(p.shape[1], dtype=np.int32) % 2])
        pos = np.concatenate([pos, p], axis=1)
        off = np.concatenate([off, [off[-1] + p.shape[1]]]).astype(np.int32)
    N, ncells = types.size, off.size - 1
    dev = torch.device("cuda")
    fused = SUS2_SH(l3k3_path, N, ["Cu", "Zr", "sus2_sh_batch_fused=1", "sus2_sh_batch_tile=256"])
    stage = SUS2_SH(l3k3_path, N, ["Cu", "Zr"])
    rng = np.random.default_rng(5)
    start = [rng.normal(size=N), rng.normal(size=3 * N), rng.normal(size=9 * N)]
    outs = []
    for pot in (fused, fused, stage):
        t = torch.as_tensor(types, device=dev)
        x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
        o = torch.as_tensor(off, device=dev)
        h = torch.as_tensor(H.reshape(-1).copy(), device=dev)
        pe, f, w = (torch.as_tensor(v, device=dev) for v in start)
        ce = torch.full((ncells,), 7.0, dtype=torch.float64, device=dev)
        cw = torch.full((9 * ncells,), 7.0, dtype=torch.float64, device=dev)
        pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce, cell_virial=cw)
        torch.cuda.synchronize()
        assert pot.sync() == 0
        outs.append([v.cpu().numpy() for v in (pe, f, w, ce, cw)])
    assert fused.info()["batch_fused"] == 1
    fused.close()
    stage.close()
    (pe1, f1, w1, ce1, cw1), (pe2, f2, w2, ce2, cw2), (pe0, f0, w0, ce0, cw0) = outs
    assert np.array_equal(pe1, pe2) and np.array_equal(ce1, ce2)
    assert np.abs(pe1 - pe0).max() < 1e-9
    assert np.sqrt(((f1 - f0) ** 2).mean()) < 1e-6 and np.sqrt(((f2 - f0) ** 2).mean()) < 1e-6
    assert np.sqrt(((w1 - w0) ** 2).mean()) < 1e-6
    assert np.abs(ce1 - ce0).max() < 1e-8 and np.abs(cw1 - cw0).max() < 1e-5
    assert ce1[-1] == 0.0 and (cw1[-9:] == 0.0).all()  # the empty cell
    # the isolated atoms' site energies are the species terms alone
    orc = O.Oracle(l3k3_path)
    for c in range(ncells):
        lo, hi = off[c], off[c + 1]
        if hi == lo:
            continue
        pe_o, f_o, _ = orc.efs(boxes[c].cpu_h, boxes[c].pbc, types[lo:hi], pos[:, lo:hi])
        assert np.abs(pe1[lo:hi] - start[0][lo:hi] - pe_o).max() < 1e-6
        fd = f1.reshape(3, N)[:, lo:hi] - start[1].reshape(3, N)[:, lo:hi]
        assert np.sqrt(((fd - f_o) ** 2).mean()) < 1e-5


@pytest.mark.parametrize("fused", [False, True], ids=["stage", "fused"])
def test_batch_neighbor_overflow_is_reported_and_recovered(l3k3_path, fused):
    """The lists are sized at the first call of a given (N, ncells); a later
    call whose cells are compressed has more neighbours than they hold.  The
    fill (the stage kernels', or the fused kernel's own) stops at the
    capacity, sus2sh_sync reports the overflow and grows the lists, and the
    next call matches the oracle."""
    off, H, boxes, types, pos = _cells([(150, 0.03, (1.0, 1.0, 1.0)), (120, 0.03, (1.1, 1.0, 0.9))], seed=81)
    N, ncells = types.size, off.size - 1
    dev = torch.device("cuda")
    pot = SUS2_SH(l3k3_path, N, ["Cu", "Zr"] + (["sus2_sh_batch_fused=1"] if fused else []))
    t = torch.as_tensor(types, device=dev)
    o = torch.as_tensor(off, device=dev)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)

    def call(scale):
        h = torch.as_tensor((H * scale).reshape(-1).copy(), device=dev)
        x = torch.as_tensor((pos * scale).reshape(-1).copy(), device=dev)
        pe, f, w, ce = z(N), z(3 * N), z(9 * N), z(ncells)
        pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce)
        torch.cuda.synchronize()
        return pot.sync(), pe.cpu().numpy(), ce.cpu().numpy()

    assert call(1.0)[0] == 0
    assert call(0.75)[0] & 1  # overflow flagged, capacity grown
    flags, pe, ce = call(0.75)
    assert flags == 0
    assert pot.info()["batch_fused"] == (1 if fused else 0)
    pot.close()
    orc = O.Oracle(l3k3_path)
    for c in range(ncells):
        lo, hi = off[c], off[c + 1]
        pe0, _, _ = orc.efs(boxes[c].cpu_h * 0.75, boxes[c].pbc, types[lo:hi], pos[:, lo:hi] * 0.75)
        scale = max(1.0, np.abs(pe0).max())
        # (FP32 bars relative to the site energies of this compressed packing)
        assert np.abs(pe[lo:hi] - pe0).max() < 1e-5 * scale
        assert abs(ce[c] - pe0.sum()) < 1e-5 * scale * (hi - lo)
