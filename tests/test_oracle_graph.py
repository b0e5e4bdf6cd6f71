"""The oracle's standard-graph builder against the reference's published
graph counts, and the product library's C++ builder against the oracle."""
import json
import os

import pytest

from sus2sh_graph import (body_lmax_from_list, build_standard_graph, explicit_metadata,
                          real_cg, clebsch_gordan, load_mtp, standard_graph_matches)

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "graph_kats.json")))


def _stats(spec):
    g = build_standard_graph(spec["l_max"], spec["k_max"], spec["body_order"],
                             body_lmax_from_list(spec["l_max"], spec["body_order"], spec["body_l_max"]))
    md = explicit_metadata(g.node_count, len(g.basic), g.products, g.scalars)
    term = md["terminal"]
    removed = sum(2 * len(t) for (_, tgt, t) in md["rows"] if term[tgt])
    remaining = dups = 0
    for (_, _, terms) in md["back"]:
        seen = set()
        for t, o, c in terms:
            if term[t]:
                continue
            remaining += 1
            if (t, o) in seen:
                dups += 1
            seen.add((t, o))
    return {
        "alpha_moments_count": g.node_count, "sh_product_count": len(g.products),
        "alpha_scalar_moments": len(g.scalars), "alpha_index_basic_count": len(g.basic),
        "tensor_blocks": len(g.tensor_blocks), "cg_blocks": g.cg_blocks, "cg_terms": g.cg_terms,
        "cg_rows": len(md["rows"]), "cg_back_rows": len(md["back"]), "layers": md["max_layer"],
        "terminal_scalars": sum(term), "removed_back_terms": removed,
        "back_terms_after_fusion": remaining, "merged_back_duplicates": dups,
    }


@pytest.mark.parametrize("name", [k for k in GOLDEN if not k.startswith("_")])
def test_published_graph_counts(name):
    kat = GOLDEN[name]
    got = _stats(kat["spec"])
    for key, want in kat.items():
        if key in ("spec", "cite"):
            continue
        assert got[key] == want, f"{name}.{key}: oracle {got[key]} != published {want} ({kat['cite']})"


def test_workload_model_counts():
    # l3k3 body-4 (the benchmark model) and l4k4 body-5 (the large model)
    s = _stats({"l_max": 3, "k_max": 3, "body_order": 4, "body_l_max": [3, 3, 3, 3]})
    assert (s["alpha_moments_count"], s["sh_product_count"], s["alpha_scalar_moments"]) == (248, 806, 107)
    assert (s["cg_rows"], s["terminal_scalars"], s["layers"]) == (200, 80, 2)
    s = _stats({"l_max": 4, "k_max": 4, "body_order": 5, "body_l_max": [4, 4, 4, 4]})
    assert (s["alpha_moments_count"], s["sh_product_count"], s["alpha_scalar_moments"]) == (5985, 33389, 2819)


def test_clebsch_gordan_identities():
    # orthonormality sum_{m1,m2} <l1 m1 l2 m2|L M><l1 m1 l2 m2|L' M'> = delta
    for l1, l2 in [(1, 1), (2, 1), (2, 2), (3, 2)]:
        for L in range(abs(l1 - l2), l1 + l2 + 1):
            for M in range(-L, L + 1):
                s = sum(clebsch_gordan(l1, m1, l2, M - m1, L, M) ** 2
                        for m1 in range(-l1, l1 + 1) if abs(M - m1) <= l2)
                assert abs(s - 1.0) < 1e-12
    # real coupling to L=0 of identical l is a scaled dot product
    for l in range(4):
        c = [[real_cg(l, a, l, b, 0, 0) for b in range(-l, l + 1)] for a in range(-l, l + 1)]
        for a in range(2 * l + 1):
            for b in range(2 * l + 1):
                if a != b:
                    assert abs(c[a][b]) < 1e-12
                else:
                    assert abs(abs(c[a][b]) - 1.0 / (2 * l + 1) ** 0.5) < 1e-12


def test_cpp_builder_matches_oracle():
    from sus2sh import standard_graph_counts
    for spec in ([3, 3, 4, None], [3, 3, 5, [3, 3, 3, 3]], [3, 3, 5, [3, 3, 2, 2]], [4, 4, 5, [4, 4, 2, 2]],
                 [2, 2, 6, None], [1, 2, 3, None], [5, 2, 4, None], [6, 2, 4, None], [6, 1, 5, None]):
        L, K, body, bl = spec
        c = standard_graph_counts(L, K, body, bl)
        g = build_standard_graph(L, K, body, body_lmax_from_list(L, body, bl) if bl else None)
        assert c["node_count"] == g.node_count
        assert c["basics"] == len(g.basic)
        assert c["products"] == len(g.products)
        assert c["scalars"] == len(g.scalars)
        assert c["tensor_blocks"] == len(g.tensor_blocks)
        assert c["cg_blocks"] == g.cg_blocks
        assert c["cg_terms"] == g.cg_terms
        assert c["max_layer"] == g.max_layer


def test_written_model_matches_standard_graph(l3k3_path, model_dir):
    # the product's writer emits exactly the oracle's standard graph
    # (validate_standard_sh_graph tolerance 2e-10 (1+|c|), sus2_sh.cu:1747-1762)
    m = load_mtp(l3k3_path)
    g = build_standard_graph(m.sh_l_max, m.sh_k_max, m.sh_body_order, m.body_lmax)
    assert standard_graph_matches(m, g)
    from sus2sh import models
    p = models.write_model(os.path.join(model_dir, "l2_b6.mtp"), l_max=2, k_max=2, body_order=6, rb_size=8,
                           seed=5)
    m = load_mtp(p)
    g = build_standard_graph(2, 2, 6)
    assert standard_graph_matches(m, g)
    # l = 6 (solid-harmonic path of the reference)
    p = models.write_model(os.path.join(model_dir, "l6_b4.mtp"), l_max=6, k_max=2, body_order=4, rb_size=8,
                           seed=6)
    m = load_mtp(p)
    assert m.sh_l_max == 6
    assert standard_graph_matches(m, build_standard_graph(6, 2, 4))
