"""ZBL short-range term on the CPU: the oracle's restatement and the engine's
pair function against the reference's own ZBL code (golden vectors written by
tests/golden/make_zbl_golden.py from src/force/sus2_zbl_common.cuh), the
reference's own unit test where the reference tree is present, the model
reader's ZBL keys, and the oracle's ZBL forces and virials against finite
differences."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import build_ref
import sus2sh_oracle as O
from sus2sh import _lib, models, structures
from sus2sh_graph import MtpError, MtpModel, load_mtp

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "zbl_kats.json")


@pytest.fixture(scope="module")
def kats():
    with open(GOLDEN) as fh:
        return json.load(fh)


def test_oracle_pair_function_matches_reference(kats):
    for zi, zj, r, inner, outer, e, de in kats["pairs"]:
        ge, gde = O.zbl_pair(zi, zj, r, inner, outer)
        assert ge == e and gde == de, (zi, zj, r, inner, outer, ge, e, gde, de)


def test_engine_pair_function_matches_reference(kats):
    lib = _lib.load()
    e, de = ctypes.c_double(), ctypes.c_double()
    for zi, zj, r, inner, outer, ge, gde in kats["pairs"]:
        assert lib.sus2sh_zbl_pair(zi, zj, r, inner, outer, ctypes.byref(e), ctypes.byref(de)) == 0
        assert e.value == ge and de.value == gde, (zi, zj, r, inner, outer)


def test_oracle_tables_match_reference(kats):
    for t in kats["tables"]:
        if t["error"] is not None:
            with pytest.raises(ValueError, match=t["error"].replace("[", r"\[").replace("]", r"\]")):
                O.zbl_tables(t["z"], t["inner"], t["outer"], t["typewise"], t["factor"])
            continue
        pin, pout = O.zbl_tables(t["z"], t["inner"], t["outer"], t["typewise"], t["factor"])
        assert list(pin) == t["inner_table"]
        assert list(pout) == t["outer_table"]
        assert list(pout * pout) == t["outer_sq"]


def test_oracle_symbols_and_radii_match_reference(kats):
    for sym, z in kats["symbols"].items():
        assert O.atomic_number(sym) == z
    lib = ctypes.CDLL(O.build_oracle())
    lib.oracle_zbl_covalent_radius.restype = ctypes.c_double
    for z, r in enumerate(kats["covalent_radius"]):
        assert lib.oracle_zbl_covalent_radius(z) == r
    d = kats["defaults"]
    assert (MtpModel.zbl_inner, MtpModel.zbl_outer, MtpModel.zbl_typewise_factor) == (d["inner"], d["outer"], d["typewise_factor"])


@pytest.mark.skipif(not build_ref.reference_present(), reason="reference tree not present")
def test_reference_unit_test_and_live_comparison():
    paths = build_ref.build()
    out = subprocess.run([paths["zbl_check"]], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and "passed" in out.stdout
    lib = ctypes.CDLL(paths["zbl_lib"])
    rng = np.random.default_rng(11)
    e, de = ctypes.c_double(), ctypes.c_double()
    for _ in range(2000):
        zi, zj = (int(v) for v in rng.integers(1, 95, size=2))
        inner = float(rng.uniform(0.0, 1.5))
        outer = inner + float(rng.uniform(0.01, 3.0))
        r = float(rng.uniform(0.0, outer * 1.1))
        lib.ref_zbl_pair(zi, zj, ctypes.c_double(r), ctypes.c_double(inner), ctypes.c_double(outer),
                         ctypes.byref(e), ctypes.byref(de))
        assert O.zbl_pair(zi, zj, r, inner, outer) == (e.value, de.value)


def _zbl_model(l3k3_path, tmp_path, name, **kw):
    return models.add_zbl(l3k3_path, str(tmp_path / name), **kw)


def test_reader_zbl_keys(l3k3_path, tmp_path):
    m = load_mtp(_zbl_model(l3k3_path, tmp_path, "a.mtp", atomic_numbers=[29, 40]))
    assert m.zbl_enabled and not m.zbl_typewise and (m.zbl_inner, m.zbl_outer) == (0.7, 1.4)
    assert m.zbl_atomic_numbers == [29, 40]
    # a factor alone switches typewise cutoffs on (sus2_sh.cu:2138-2140)
    m = load_mtp(_zbl_model(l3k3_path, tmp_path, "b.mtp", factor=1.1, outer=3.0))
    assert m.zbl_typewise and m.zbl_typewise_factor == 1.1 and m.zbl_outer == 3.0
    m = load_mtp(_zbl_model(l3k3_path, tmp_path, "c.mtp", factor=1.1, typewise=False))
    assert not m.zbl_typewise
    m = load_mtp(_zbl_model(l3k3_path, tmp_path, "d.mtp", enabled="off"))
    assert not m.zbl_enabled
    with pytest.raises(MtpError, match="boolean"):
        load_mtp(_zbl_model(l3k3_path, tmp_path, "e.mtp", enabled="On"))


def test_engine_rejects_bad_zbl_metadata(l3k3_path, tmp_path):
    lib = _lib.load()
    h = ctypes.c_void_p()
    path = _zbl_model(l3k3_path, tmp_path, "nosym.mtp")
    assert lib.sus2sh_create(path.encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "requires zbl_atomic_numbers" in lib.sus2sh_last_error().decode()
    opts = (ctypes.c_char_p * 2)(b"Cu", b"Xx")
    assert lib.sus2sh_create(path.encode(), 0, 2, ctypes.cast(opts, ctypes.c_void_p), ctypes.byref(h)) == -1
    assert "cannot map element symbol" in lib.sus2sh_last_error().decode()
    path = _zbl_model(l3k3_path, tmp_path, "three.mtp", atomic_numbers=[29, 40, 13])
    assert lib.sus2sh_create(path.encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "one atomic number per species" in lib.sus2sh_last_error().decode()
    path = _zbl_model(l3k3_path, tmp_path, "badcut.mtp", atomic_numbers=[29, 40], inner=1.5, outer=1.4)
    assert lib.sus2sh_create(path.encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "inner < outer" in lib.sus2sh_last_error().decode()
    path = _zbl_model(l3k3_path, tmp_path, "badz.mtp", atomic_numbers=[29, 95], factor=0.7)
    assert lib.sus2sh_create(path.encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "[1, 94]" in lib.sus2sh_last_error().decode()


def test_oracle_two_atom_energy_is_sus2_plus_pair(l3k3_path, tmp_path):
    path = _zbl_model(l3k3_path, tmp_path, "pair.mtp", atomic_numbers=[29, 40], inner=1.0, outer=3.0)
    box = np.diag([40.0, 40.0, 40.0]).ravel()
    pbc = np.array([0, 0, 0], dtype=np.int32)
    types = np.array([0, 1], dtype=np.int32)
    pos = np.array([[10.0, 12.4], [10.0, 10.3], [10.0, 9.7]])
    r = float(np.linalg.norm(pos[:, 1] - pos[:, 0]))
    plain = O.Oracle(l3k3_path).efs(box, pbc, types, pos)
    zbl = O.Oracle(path).efs(box, pbc, types, pos)
    e, de = O.zbl_pair(29, 40, r, 1.0, 3.0)
    assert e > 0
    assert np.allclose(zbl[0] - plain[0], [0.5 * e, 0.5 * e], rtol=0, atol=1e-13 * e)
    u = (pos[:, 1] - pos[:, 0]) / r
    assert np.allclose(zbl[1][:, 0] - plain[1][:, 0], de * u, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("kw", [dict(atomic_numbers=[29, 40], inner=1.0, outer=3.0),
                                dict(atomic_numbers=[29, 40], factor=1.2, outer=3.5)])
def test_oracle_zbl_forces_and_virial(l3k3_path, tmp_path, kw):
    orc = O.Oracle(_zbl_model(l3k3_path, tmp_path, "fd.mtp", **kw))
    box, types, pos = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.15, seed=9)
    pe, f, v = orc.efs(box.cpu_h, box.pbc, types, pos)
    hstep = 1e-5
    rng = np.random.default_rng(2)
    for i in rng.choice(types.size, 4, replace=False):
        for a in range(3):
            p1 = pos.copy(); p1[a, i] += hstep
            p2 = pos.copy(); p2[a, i] -= hstep
            fd = -(orc.efs(box.cpu_h, box.pbc, types, p1)[0].sum()
                   - orc.efs(box.cpu_h, box.pbc, types, p2)[0].sum()) / (2 * hstep)
            assert abs(fd - f[a, i]) < 1e-6 * max(1.0, abs(f[a, i]))
    # virial: sum_i W_i^{ab} = -dE/de_ab under x -> (1 + e) x
    H = box.cpu_h.reshape(3, 3)
    for a, b, q in ((0, 0, 0), (1, 1, 1), (0, 1, 3), (2, 0, 7)):
        E = []
        for sgn in (1, -1):
            D = np.eye(3)
            D[a, b] += sgn * hstep
            E.append(orc.efs((D @ H).ravel(), box.pbc, types, D @ pos)[0].sum())
        assert abs(-(E[0] - E[1]) / (2 * hstep) - v[q].sum()) < 1e-6 * max(1.0, abs(v[q].sum()))
