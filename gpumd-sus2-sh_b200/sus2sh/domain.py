"""Spatial decomposition of one periodic box over ranks (one GPU each).

The path is short-ranged, so it shards by space: slabs along the box axis of
largest thickness.  Rank r owns the atoms whose fractional coordinate along
that axis lies in [r/R, (r+1)/R).  Its local system is its owned atoms plus
ghosts: copies of the atoms of the neighbouring slabs within ``halo``
(the cutoff, plus the Verlet skin when lists are reused) of its two faces,
with the periodic images across the box made explicit, so the slab axis is
open in the local system and the other axes keep the box's periodicity.

Only owned atoms are centres.  With the engine's explicit adjoint
(``sus2sh_forward``, then ``sus2sh_backward`` with per-atom energy weights
w = 1 on owned atoms and 0 on ghosts) a rank gets the site energies and
per-atom virials of its owned atoms and the forces of those energies on every
local atom; the virial of an edge belongs to its centre, so ghosts carry
none.  The forces on ghosts are sent back to their owners and added there
(the reverse halo exchange), and the total energy and virial are FP64
all-reduced.  The result equals the one-box evaluation: each site energy is
computed once, by its owner, from its complete neighbourhood.

Requirements: every slab at least ``halo`` thick (so ghosts come from the two
adjacent slabs only), and R >= 2 only along a periodic axis.  The exchange
uses torch.distributed point-to-point messages between those neighbours (NCCL
between GPUs; gloo in the CPU tests).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def thicknesses(h) -> np.ndarray:
    """Distance between the opposite faces of the cell along each box vector
    (h row-major, the box vectors as columns)."""
    m = np.asarray(h, dtype=np.float64).reshape(3, 3)
    vol = abs(np.linalg.det(m))
    out = np.zeros(3)
    for d in range(3):
        a, b = m[:, (d + 1) % 3], m[:, (d + 2) % 3]
        out[d] = vol / np.linalg.norm(np.cross(a, b))
    return out


@dataclass
class SlabDomain:
    rank: int
    nranks: int
    axis: int
    owned: np.ndarray        # global indices of the owned atoms (ascending)
    ghosts: np.ndarray       # global index of each ghost (an atom may be the ghost of both faces)
    ghost_shift: np.ndarray  # (3, n_ghosts) Cartesian image shift added to each ghost's position
    ghost_owner: np.ndarray  # rank owning each ghost
    h: np.ndarray            # (9,) the box
    pbc: np.ndarray          # (3,) the box's periodicity, the slab axis open when nranks > 1

    @property
    def n_local(self) -> int:
        return self.owned.size + self.ghosts.size

    def center_mask(self) -> np.ndarray:
        """1 on owned atoms, 0 on ghosts (local order: owned, then ghosts)."""
        return np.concatenate([np.ones(self.owned.size), np.zeros(self.ghosts.size)])

    def local_types(self, types) -> np.ndarray:
        types = np.asarray(types)
        return np.concatenate([types[self.owned], types[self.ghosts]]).astype(np.int32)

    def local_positions(self, pos) -> np.ndarray:
        pos = np.asarray(pos, dtype=np.float64)
        return np.ascontiguousarray(np.concatenate([pos[:, self.owned], pos[:, self.ghosts] + self.ghost_shift],
                                                   axis=1))


def slab_partition(h, pbc, pos, nranks: int, halo: float, axis: int | None = None) -> list[SlabDomain]:
    """The R = nranks slab domains of a box (h, pbc) with positions (3, N)."""
    m = np.asarray(h, dtype=np.float64).reshape(3, 3)
    pbc = np.asarray(pbc, dtype=np.int32).reshape(3)
    pos = np.asarray(pos, dtype=np.float64)
    N = pos.shape[1]
    if nranks == 1:
        return [SlabDomain(0, 1, 0, np.arange(N), np.zeros(0, dtype=np.int64), np.zeros((3, 0)),
                           np.zeros(0, dtype=np.int64), m.reshape(9).copy(), pbc.copy())]
    th = thicknesses(m)
    if axis is None:
        cand = [d for d in range(3) if pbc[d]]
        if not cand:
            raise ValueError("slab decomposition needs a periodic axis")
        axis = max(cand, key=lambda d: th[d])
    if not pbc[axis]:
        raise ValueError("the slab axis must be periodic")
    if th[axis] / nranks < halo:
        raise ValueError(f"slabs of {th[axis] / nranks:.3f} A are thinner than the halo of {halo:.3f} A")
    s = np.linalg.solve(m, pos)[axis]
    s = s - np.floor(s)
    slab = np.minimum((s * nranks).astype(np.int64), nranks - 1)
    hf = halo / th[axis]
    shift_vec = m[:, axis]
    local_pbc = pbc.copy()
    local_pbc[axis] = 0
    out = []
    for r in range(nranks):
        lo, hi = r / nranks, (r + 1) / nranks
        owned = np.nonzero(slab == r)[0]
        gi, gs, go = [], [], []
        for n in (-1, 0, 1):
            sp = s + n
            near = ((sp >= lo - hf) & (sp < lo)) | ((sp >= hi) & (sp < hi + hf))
            idx = np.nonzero(near)[0]
            gi.append(idx)
            gs.append(np.repeat(n, idx.size))
            go.append(slab[idx])
        gi, gs, go = np.concatenate(gi), np.concatenate(gs), np.concatenate(go)
        order = np.lexsort((gs, gi))
        gi, gs, go = gi[order], gs[order], go[order]
        out.append(SlabDomain(r, nranks, axis, owned, gi, np.outer(shift_vec, gs), go, m.reshape(9).copy(),
                              local_pbc))
    return out


def reverse_add_forces(dom: SlabDomain, f_local: np.ndarray, dist=None, group=None) -> np.ndarray:
    """Forces on the owned atoms (3, n_owned): the local forces of the owned
    atoms plus the ghost forces the other ranks computed for them.  Ghost
    forces travel to their owners as (global index, force) messages,
    point-to-point with every rank that shares ghosts (the adjacent slabs)."""
    import torch
    if dist is None:
        import torch.distributed as dist
    no = dom.owned.size
    f_local = np.asarray(f_local, dtype=np.float64).reshape(3, dom.n_local)
    out = f_local[:, :no].copy()
    if dom.nranks == 1:
        return out
    fg = f_local[:, no:]
    peers = sorted({(dom.rank - 1) % dom.nranks, (dom.rank + 1) % dom.nranks} - {dom.rank})
    sends, counts_in = [], {}
    for q in peers:
        sel = dom.ghost_owner == q
        idx = torch.as_tensor(dom.ghosts[sel].astype(np.int64))
        val = torch.as_tensor(np.ascontiguousarray(fg[:, sel].T))  # (n, 3)
        sends.append((q, idx, val))
    # sizes first, then indices and forces; every rank posts its sends before
    # its receives, so no pair of ranks waits on each other
    reqs = []
    for q, idx, _ in sends:
        reqs.append(dist.isend(torch.tensor([idx.numel()], dtype=torch.int64), q, group=group, tag=1))
    for q in peers:
        n = torch.zeros(1, dtype=torch.int64)
        dist.recv(n, q, group=group, tag=1)
        counts_in[q] = int(n.item())
    for r_ in reqs:
        r_.wait()
    reqs = []
    for q, idx, val in sends:
        reqs.append(dist.isend(idx, q, group=group, tag=2))
        reqs.append(dist.isend(val, q, group=group, tag=3))
    for q in peers:
        idx = torch.zeros(counts_in[q], dtype=torch.int64)
        val = torch.zeros((counts_in[q], 3), dtype=torch.float64)
        dist.recv(idx, q, group=group, tag=2)
        dist.recv(val, q, group=group, tag=3)
        pos_in_owned = np.searchsorted(dom.owned, idx.numpy())
        if idx.numel() and not np.array_equal(dom.owned[pos_in_owned], idx.numpy()):
            raise RuntimeError("ghost force for an atom this rank does not own")
        np.add.at(out.T, pos_in_owned, val.numpy())
    for r_ in reqs:
        r_.wait()
    return out


def allreduce_sum(values, dist=None, group=None) -> np.ndarray:
    """FP64 all-reduce (sum) of a small vector: the energy and the 3x3 virial."""
    import torch
    if dist is None:
        import torch.distributed as dist
    t = torch.as_tensor(np.asarray(values, dtype=np.float64).copy())
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.numpy()


def engine_evaluator(pot, device="cuda"):
    """Local evaluation through the engine's explicit adjoint: forward, then
    backward with the centre mask as per-atom energy weights.  Returns a
    callable (dom, types, pos) -> (pe[n_local], f[3, n_local], w[9, n_local])
    on the host; pe and w are zero on ghosts."""
    import torch

    from .potential import Box

    def run(dom: SlabDomain, types, pos):
        n = dom.n_local
        dev = torch.device(device)
        box = Box(dom.h, dom.pbc)
        t = torch.as_tensor(dom.local_types(types), device=dev)
        x = torch.as_tensor(dom.local_positions(pos).reshape(-1), device=dev)
        mask = torch.as_tensor(dom.center_mask(), device=dev)
        pe = torch.zeros(n, dtype=torch.float64, device=dev)
        g = torch.zeros(3 * n, dtype=torch.float64, device=dev)
        w = torch.zeros(9 * n, dtype=torch.float64, device=dev)
        pot.forward(box, t, x, pe)
        pot.backward(mask, g, w)
        torch.cuda.synchronize()
        return ((pe * mask).cpu().numpy(), -g.view(3, n).cpu().numpy(), w.view(9, n).cpu().numpy())

    return run
