"""Saved product graphs that fail the standard-graph match.

The reference runs such a file's own product list through its explicit
metadata path (``standard_sh_graph_matches`` false, ``src/force/sus2_sh.cu:
1872-1911,2095-2103``): trainer-pruned ("q-total") graphs and hand-edited ones.
The engine always runs the file's own product list.  Each file here is
derived from a standard model (``tests/graph_edit.py``): scalars pruned with
the products only they needed, or coefficients scaled, extra basic x basic
terms added to intermediate rows and the rows reordered.  The engine is
compared with the FP64 oracle and with the reference's own engine
(``oracle/_ref/ref_sus2sh``), whose loader reports the explicit mode for each.

Bars: FP64 engine vs oracle 1e-9 (relative to the site-energy scale for the
body-5 model); FP32 engine vs oracle and vs the reference's FP64 path 1e-6
eV/site and 1e-5 eV/A force RMS for the l3k3 graphs, the same bars relative to
the energy and force scales for the body-5 graphs (site energies of tens of
eV); the reference's FP64 forces carry its FP32 scatter buffers (1e-6 of the
largest force).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import graph_edit  # noqa: E402
import ref_engine  # noqa: E402
import sus2sh_oracle as O  # noqa: E402
from sus2sh import models, structures  # noqa: E402
from test_parity_gpu import engine_efs  # noqa: E402


def _variants(src, d, tag):
    text = open(src).read()
    out = {}
    p = os.path.join(d, f"{tag}_pruned.mtp")
    open(p, "w").write(graph_edit.prune(text, lambda s, body: body <= 3 or s % 3 == 0))
    out["pruned"] = p
    p = os.path.join(d, f"{tag}_edited.mtp")
    open(p, "w").write(graph_edit.edit(text, seed=3))
    out["edited"] = p
    return out


def _scales(pe, f):
    return max(1.0, float(np.abs(pe).max())), max(1.0, float(np.sqrt((f ** 2).mean())))


def _check(path, box, types, pos, relative):
    orc = O.Oracle(path)
    pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types, pos)
    es, fs = _scales(pe0, f0) if relative else (1.0, 1.0)
    pe, f, w = engine_efs(path, box, types, pos, ("sus2_float=0",))
    assert np.abs(pe - pe0).max() / es < 1e-9 and np.abs(f - f0).max() / fs < 1e-8
    pe, f, w = engine_efs(path, box, types, pos)
    assert np.abs(pe - pe0).max() / es < 1e-6 * (5 if relative else 1)
    assert np.sqrt(((f - f0) ** 2).mean()) / fs < 1e-5
    if ref_engine.available():
        r = ref_engine.run(path, box.cpu_h, box.pbc, types, pos, ("Cu", "Zr", "sus2_float=0"))
        assert "mode=explicit" in r[4]
        pe_r, f_r = r[0], r[1]
        # against the oracle with the reference's FP32-rounded radial tables
        pe_rr, f_rr, _ = O.Oracle(path, reference_rounding=True).efs(box.cpu_h, box.pbc, types, pos)
        assert np.abs(pe_r - pe_rr).max() / es < 1e-9
        assert np.abs(f_r - f_rr).max() < 1e-6 * max(1.0, np.abs(f_rr).max())
        assert np.abs(pe - pe_r).max() / es < 1e-6 * (5 if relative else 1)
        assert np.sqrt(((f - f_r) ** 2).mean()) / fs < 1e-5


@pytest.mark.parametrize("kind", ["pruned", "edited"])
def test_l3k3_explicit_graphs(l3k3_path, tmp_path, kind):
    path = _variants(l3k3_path, str(tmp_path), "l3k3")[kind]
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.5, 0.5), 0.05, seed=31)
    _check(path, box, types, pos, relative=False)
    box, types, pos = structures.fcc(3, 3, 3, 3.8, (0.5, 0.5), 0.1, seed=32)  # explicit images
    _check(path, box, types, pos, relative=False)


@pytest.mark.parametrize("kind", ["pruned", "edited"])
def test_body5_explicit_graphs_component_split_kernel(tmp_path, kind):
    # l3k3 body 5 (5,475 products): above the single-function limit, so the
    # engine runs the component-split kernel on the saved graph
    src = models.write_model(str(tmp_path / "l3k3b5.mtp"), l_max=3, k_max=3, body_order=5, seed=55)
    path = _variants(src, str(tmp_path), "l3k3b5")[kind]
    box, types, pos = structures.fcc(5, 5, 5, 3.8, (0.5, 0.5), 0.05, seed=33)
    _check(path, box, types, pos, relative=True)
    from sus2sh import SUS2_SH
    pot = SUS2_SH(path, types.size, ["Cu", "Zr"])
    info = pot.info()
    pot.close()
    assert info["standard_graph_matched"] == 0


def test_q_total_option_on_a_standard_file(l3k3_path):
    # the reference's sus2_factor_pruning=q-total forces its explicit path on
    # a standard file; the engine accepts the option and gives the same result
    box, types, pos = structures.fcc(4, 4, 4, 3.8, (0.5, 0.5), 0.05, seed=34)
    pe, f, _ = engine_efs(l3k3_path, box, types, pos, ("sus2_factor_pruning=q-total", "sus2_float=0"))
    pe0, f0, _ = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, pos)
    assert np.abs(pe - pe0).max() < 1e-9
    if ref_engine.available():
        r = ref_engine.run(l3k3_path, box.cpu_h, box.pbc, types, pos,
                           ("Cu", "Zr", "sus2_float=0", "sus2_factor_pruning=q-total"))
        assert "factor_pruning=q-total, mode=explicit" in r[4]
        pe_rr, _, _ = O.Oracle(l3k3_path, reference_rounding=True).efs(box.cpu_h, box.pbc, types, pos)
        assert np.abs(r[0] - pe_rr).max() < 1e-9
