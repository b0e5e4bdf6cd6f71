"""Spatial decomposition (sus2sh/domain.py) on CPU ranks.

Each rank evaluates its slab's local system (owned atoms as centres, ghosts
within the cutoff, the slab axis open) with the FP64 oracle restricted to the
owned centres, sends the forces on its ghosts to their owners over gloo, and
all-reduces energy and virial in FP64.  The gathered result must equal the
one-box oracle evaluation of the periodic box (per-atom energies, forces,
virials, totals) to 1e-10.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sus2sh import domain, structures  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(name):
    if name == "cube":
        return structures.fcc(6, 6, 6, 3.8, (0.5, 0.5), 0.1, seed=71)
    if name == "long":
        return structures.fcc(8, 3, 3, 3.8, (0.6, 0.4), 0.1, seed=72)
    box, types, pos = structures.fcc(6, 4, 4, 3.8, (0.5, 0.5), 0.08, seed=73)  # triclinic
    h = np.array([[22.8, 2.1, -1.3], [0.0, 15.2, 1.7], [0.0, 0.0, 15.2]])
    frac = np.linalg.solve(box.cpu_h.reshape(3, 3), pos)
    from sus2sh import Box
    return Box(h.ravel()), types, h @ frac


def _rank_main(rank, world, port, model, case, out_dir):
    import sys
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "gpumd-sus2-sh_b200"))
    import torch.distributed as dist

    import sus2sh_oracle as O
    from sus2sh import domain as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        box, types, pos = _case(case)
        orc = O.Oracle(model)
        dom = D.slab_partition(box.cpu_h, box.pbc, pos, world, orc.model.max_dist)[rank]
        pe, f, w = orc.efs_centers(dom.h, dom.pbc, dom.local_types(types), dom.local_positions(pos),
                                   dom.center_mask())
        f_owned = D.reverse_add_forces(dom, f)
        no = dom.owned.size
        totals = D.allreduce_sum(np.concatenate([[pe[:no].sum()], w[:, :no].sum(axis=1)]))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), owned=dom.owned, pe=pe[:no], f=f_owned, w=w[:, :no],
                 totals=totals, ghosts=dom.ghosts.size)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [(2, "cube"), (2, "triclinic"), (3, "long")])
def test_slab_ranks_match_one_box(l3k3_path, world, case):
    import torch.multiprocessing as mp
    import sus2sh_oracle as O
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), l3k3_path, case, d), nprocs=world, join=True,
                           start_method="spawn")
        parts = [np.load(os.path.join(d, f"rank{r}.npz")) for r in range(world)]
    box, types, pos = _case(case)
    N = types.size
    pe0, f0, w0 = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, pos)
    owned = np.concatenate([p["owned"] for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(N))  # every atom owned once
    assert all(p["ghosts"] > 0 for p in parts)
    pe = np.zeros(N)
    f = np.zeros((3, N))
    w = np.zeros((9, N))
    for p in parts:
        pe[p["owned"]] = p["pe"]
        f[:, p["owned"]] = p["f"]
        w[:, p["owned"]] = p["w"]
    assert np.abs(pe - pe0).max() < 1e-10
    assert np.abs(f - f0).max() < 1e-10
    assert np.abs(w - w0).max() < 1e-9
    for p in parts:  # the all-reduced totals, on every rank
        assert abs(p["totals"][0] - pe0.sum()) < 1e-8
        assert np.abs(p["totals"][1:] - w0.sum(axis=1)).max() < 1e-8


def test_partition_geometry():
    box, types, pos = _case("long")
    rc = 5.0
    doms = domain.slab_partition(box.cpu_h, box.pbc, pos, 4, rc)
    assert doms[0].axis == 0 and all(d.pbc[0] == 0 and d.pbc[1] == 1 for d in doms)
    assert sum(d.owned.size for d in doms) == types.size
    L = box.cpu_h[0]
    for d in doms:
        lo, hi = d.rank * L / 4, (d.rank + 1) * L / 4
        xo = d.local_positions(pos)[0, :d.owned.size]
        xg = d.local_positions(pos)[0, d.owned.size:]
        assert np.all((np.mod(xo, L) >= lo - 1e-9) & (np.mod(xo, L) < hi + 1e-9))
        assert np.all(((xg >= lo - rc) & (xg < lo)) | ((xg >= hi) & (xg < hi + rc)))
        assert set(d.ghost_owner) <= {(d.rank - 1) % 4, (d.rank + 1) % 4}
    with pytest.raises(ValueError):
        domain.slab_partition(box.cpu_h, box.pbc, pos, 8, rc)  # 3.8 A slabs: thinner than the halo
