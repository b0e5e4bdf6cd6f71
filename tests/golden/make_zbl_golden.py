"""Generates ``zbl_kats.json``: outputs of the reference's own ZBL code
(src/force/sus2_zbl_common.cuh, compiled by ``oracle/build_ref.py`` into
``oracle/_ref/libref_zbl.so``) on a fixed set of inputs.  Run from the repo
root in a checkout next to the reference tree:

    python tests/golden/make_zbl_golden.py
"""
from __future__ import annotations

import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build_ref  # noqa: E402

# (zi, zj) pairs: H-C of the reference's unit test, the benchmark's Cu/Zr/Al,
# and the table ends
PAIRS = [(1, 6), (6, 1), (29, 29), (29, 40), (40, 40), (13, 29), (1, 1), (94, 94), (8, 74)]
# (inner, outer) cutoffs: the defaults and wider ones the tests' models use
CUTS = [(0.7, 1.4), (1.0, 3.0), (0.0, 2.3), (0.5, 5.5)]
RS = [0.05, 0.3, 0.69999, 0.7, 0.70001, 0.9, 1.0, 1.2, 1.39999, 1.4, 1.6, 2.0, 2.29999, 2.9, 3.5, 5.4999]
TABLES = [
    dict(z=[1, 6], inner=0.7, outer=1.4, typewise=1, factor=0.7),
    dict(z=[29, 40], inner=0.7, outer=1.4, typewise=0, factor=0.0),
    dict(z=[29, 40], inner=1.0, outer=3.0, typewise=0, factor=0.0),
    dict(z=[29, 40, 13], inner=0.7, outer=3.5, typewise=1, factor=1.2),
    dict(z=[29, 40, 13], inner=0.7, outer=2.5, typewise=1, factor=1.2),
    dict(z=[94, 1], inner=0.7, outer=9.0, typewise=1, factor=0.5),
    # failing checks (reference messages)
    dict(z=[], inner=0.7, outer=1.4, typewise=0, factor=0.0),
    dict(z=[29], inner=-0.1, outer=1.4, typewise=0, factor=0.0),
    dict(z=[29], inner=0.7, outer=0.0, typewise=0, factor=0.0),
    dict(z=[29], inner=0.7, outer=1.4, typewise=1, factor=0.4),
    dict(z=[29], inner=1.4, outer=1.4, typewise=0, factor=0.0),
    dict(z=[29, 0], inner=0.7, outer=1.4, typewise=0, factor=0.0),
    dict(z=[29, 95], inner=0.7, outer=1.4, typewise=1, factor=0.7),
    dict(z=[29, 95], inner=0.7, outer=1.4, typewise=0, factor=0.0),
]
SYMBOLS = ["H", "C", "Cl", "Co", "Cu", "Zr", "Al", "Pu", "W", "Xx", "cu", ""]


def main() -> None:
    paths = build_ref.build()
    lib = ctypes.CDLL(paths["zbl_lib"])
    lib.ref_zbl_covalent_radius.restype = ctypes.c_double
    lib.ref_zbl_typewise_outer.restype = ctypes.c_double
    e, de = ctypes.c_double(), ctypes.c_double()
    pairs = []
    for zi, zj in PAIRS:
        for inner, outer in CUTS:
            for r in RS:
                lib.ref_zbl_pair(zi, zj, ctypes.c_double(r), ctypes.c_double(inner), ctypes.c_double(outer),
                                 ctypes.byref(e), ctypes.byref(de))
                pairs.append([zi, zj, r, inner, outer, e.value, de.value])
    tables = []
    for t in TABLES:
        S = len(t["z"])
        zarr = (ctypes.c_int * max(S, 1))(*t["z"])
        pin = (ctypes.c_double * max(S * S, 1))()
        pout = (ctypes.c_double * max(S * S, 1))()
        psq = (ctypes.c_double * max(S * S, 1))()
        err = ctypes.create_string_buffer(256)
        ok = lib.ref_zbl_tables(S, zarr, ctypes.c_double(t["inner"]), ctypes.c_double(t["outer"]), t["typewise"],
                                ctypes.c_double(t["factor"]), pin, pout, psq, err, 256)
        rec = dict(t)
        if ok:
            rec.update(inner_table=list(pin)[:S * S], outer_table=list(pout)[:S * S],
                       outer_sq=list(psq)[:S * S], error=None)
        else:
            rec.update(error=err.value.decode())
        tables.append(rec)
    inner, outer, factor = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib.ref_zbl_defaults(ctypes.byref(inner), ctypes.byref(outer), ctypes.byref(factor))
    out = dict(
        source="src/force/sus2_zbl_common.cuh via oracle/ref_zbl_harness.cpp",
        defaults=dict(inner=inner.value, outer=outer.value, typewise_factor=factor.value),
        covalent_radius=[lib.ref_zbl_covalent_radius(z) for z in range(0, 96)],
        symbols={s: lib.ref_zbl_atomic_number(s.encode()) for s in SYMBOLS},
        pairs=pairs,
        tables=tables,
    )
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "zbl_kats.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
        fh.write("\n")
    print(path, len(pairs), "pairs", len(tables), "tables")


if __name__ == "__main__":
    main()
