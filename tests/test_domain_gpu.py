"""The engine as the per-rank evaluator of the spatial decomposition.

Each slab's local system (owned atoms as centres, ghosts within the cutoff,
the slab axis open) goes through sus2sh_forward and sus2sh_backward with the
centre mask as per-atom energy weights (sus2sh.domain.engine_evaluator).  The
slabs run one after another in this process on one GPU, and the reverse halo
exchange is done on the host by global index, as the ranks' messages would do
it.  The result must equal the engine's and the oracle's one-box evaluation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import SUS2_SH, domain, structures  # noqa: E402
from test_parity_gpu import engine_efs  # noqa: E402


@pytest.mark.parametrize("nranks", [2, 4])
@pytest.mark.parametrize("fp64", [False, True])
def test_slabs_on_the_engine_match_one_box(l3k3_path, nranks, fp64):
    box, types, pos = structures.fcc(12, 6, 6, 3.8, (0.6, 0.4), 0.08, seed=81)
    N = types.size
    opts = ["Cu", "Zr"] + (["sus2_float=0"] if fp64 else [])
    doms = domain.slab_partition(box.cpu_h, box.pbc, pos, nranks, 5.0)
    pe = np.zeros(N)
    f = np.zeros((3, N))
    w = np.zeros((9, N))
    for d in doms:
        pot = SUS2_SH(l3k3_path, d.n_local, opts)
        pe_l, f_l, w_l = domain.engine_evaluator(pot)(d, types, pos)
        pot.close()
        no = d.owned.size
        pe[d.owned] = pe_l[:no]
        w[:, d.owned] = w_l[:, :no]
        np.add.at(f.T, d.owned, f_l[:, :no].T)
        np.add.at(f.T, d.ghosts, f_l[:, no:].T)  # reverse halo exchange
        assert np.all(pe_l[no:] == 0.0) and np.all(w_l[:, no:] == 0.0)
    pe1, f1, w1 = engine_efs(l3k3_path, box, types, pos, opts[2:])
    pe0, f0, w0 = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, pos)
    if fp64:
        assert np.abs(pe - pe1).max() < 1e-10 and np.abs(f - f1).max() < 1e-10 and np.abs(w - w1).max() < 1e-9
        assert np.abs(pe - pe0).max() < 1e-9 and np.abs(f - f0).max() < 1e-9
    else:
        assert np.abs(pe - pe0).max() < 1e-6 and np.sqrt(((f - f0) ** 2).mean()) < 1e-5
        assert np.sqrt(((w - w0) ** 2).mean()) < 1e-5
        assert np.abs(pe - pe1).max() < 1e-6
