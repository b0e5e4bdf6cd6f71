"""Saved product graphs that are not the standard graph, for tests.

The reference compares a model file's ``sh_products`` / ``alpha_moment_mapping``
with the standard real-CG graph it would build (``standard_sh_graph_matches``,
``src/force/sus2_sh.cu:1872-1911``) and, when they differ, runs the file's own
product list through its explicit metadata path (``:2095-2103``; the route of
trainer-pruned "q-total" graphs, ``docs/gpumd-sus2-sh-interface-plan.md:1995``).
These helpers derive such files from a standard model's text:

* ``prune``: keep a subset of the scalar moments and drop every product that
  no kept scalar needs (a pruned graph with unused moment slots, as a
  trainer's q-total pruning leaves);
* ``edit``: scale some product coefficients, add extra terms to some
  intermediate rows, and reorder the list row by row (still topological).
"""
from __future__ import annotations

import re

import numpy as np


def _list(text: str, key: str) -> str:
    m = re.search(r"^" + key + r" = \{(.*)\}$", text, flags=re.M)
    assert m, key
    return m.group(1)


def _set(text: str, key: str, body: str) -> str:
    return re.sub(r"^" + key + r" = \{.*\}$", lambda _: f"{key} = {{{body}}}", text, count=1, flags=re.M)


def _set_count(text: str, key: str, value: int) -> str:
    return re.sub(r"^(\s*" + key + r" = )\S+$", lambda mm: mm.group(1) + str(value), text, count=1, flags=re.M)


def parse(text: str):
    prods = [(int(a), int(b), int(t), float(c)) for a, b, t, c in
             re.findall(r"\{(-?\d+), (-?\d+), (-?\d+), ([^}]+)\}", _list(text, "sh_products"))]
    mapping = [int(x) for x in _list(text, "alpha_moment_mapping").split(",")]
    coeffs = [float(x) for x in _list(text, "moment_coeffs").split(",")]
    info = re.findall(r"\{(\d+)\}", _list(text, "sh_scalar_info"))
    basics = int(re.search(r"^alpha_index_basic_count = (\d+)$", text, flags=re.M).group(1))
    return prods, mapping, coeffs, [int(x) for x in info], basics


def write(text: str, prods, mapping, coeffs, info) -> str:
    text = _set(text, "sh_products", ", ".join(f"{{{a}, {b}, {t}, {c!r}}}" for a, b, t, c in prods))
    text = _set_count(text, "sh_product_count", len(prods))
    text = _set(text, "alpha_moment_mapping", ", ".join(str(x) for x in mapping))
    text = _set_count(text, "alpha_scalar_moments", len(mapping))
    text = _set(text, "moment_coeffs", ", ".join(repr(x) for x in coeffs))
    text = _set(text, "sh_scalar_info", ", ".join(f"{{{x}}}" for x in info))
    text = _set_count(text, "sh_scalar_info_count", len(info))
    return text


def prune(text: str, keep) -> str:
    """Keeps the scalars s with keep(s, body_order) true and the products
    they need."""
    prods, mapping, coeffs, info, _ = parse(text)
    kept = [s for s in range(len(mapping)) if keep(s, info[s])]
    need = {mapping[s] for s in kept}
    rows = {}
    for p in prods:
        rows.setdefault(p[2], []).append(p)
    for t in sorted(rows, reverse=True):  # targets are defined before use: walk back
        if t in need:
            for a, b, _, _ in rows[t]:
                need.add(a)
                need.add(b)
    out = [p for p in prods if p[2] in need]
    return write(text, out, [mapping[s] for s in kept], [coeffs[s] for s in kept], [info[s] for s in kept])


def edit(text: str, seed: int = 0, scale_fraction: float = 0.1, extra_rows: int = 12) -> str:
    """Scales a fraction of the coefficients by (1 + U(-0.3, 0.3)), adds one
    basic x basic term to `extra_rows` intermediate rows, and writes the
    products grouped by target in descending row order of first use where
    that keeps the list topological (otherwise in file order)."""
    rng = np.random.default_rng(seed)
    prods, mapping, coeffs, info, nb = parse(text)
    prods = [(a, b, t, c * (1.0 + rng.uniform(-0.3, 0.3)) if rng.random() < scale_fraction else c)
             for a, b, t, c in prods]
    rows, order = {}, []
    for p in prods:
        if p[2] not in rows:
            rows[p[2]] = []
            order.append(p[2])
        rows[p[2]].append(p)
    inter = [t for t in order if all(a < nb and b < nb for a, b, _, _ in rows[t])]
    for t in rng.choice(inter, size=min(extra_rows, len(inter)), replace=False):
        a, b = sorted(int(x) for x in rng.integers(0, nb, size=2))
        rows[int(t)].insert(0, (a, b, int(t), float(rng.normal(0.0, 0.05))))
    # rows whose operands are all basics first (reversed among themselves),
    # then the others in their original order: a different, still
    # topological, order of the rows
    first = [t for t in order if all(a < nb and b < nb for a, b, _, _ in rows[t])][::-1]
    rest = [t for t in order if t not in set(first)]
    out = [p for t in first + rest for p in rows[t]]
    return write(text, out, mapping, coeffs, info)
