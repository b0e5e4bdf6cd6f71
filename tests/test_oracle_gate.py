"""Two-layer mu-body gate models on the CPU: the readers (engine and oracle)
against the reference loader's checks and messages (src/force/sus2_sh.cu:
2153-2268, 2354-2378, 2412-2461), and the oracle's gate forces and virials
against finite differences of its energy (they pin the whole chain: gate
signals, tanh multipliers, dE/dh accumulation, gate back-propagation and the
first-layer force pass)."""
import ctypes
import re

import numpy as np
import pytest

import sus2sh_oracle as O
from sus2sh import _lib, models, structures
from sus2sh_graph import MtpError, load_mtp


@pytest.fixture(scope="module", params=["mu-scalar-full", "mu-body-linear-combo"])
def gate_model(request, l3k3_path, model_dir):
    return models.add_gate(l3k3_path, f"{model_dir}/gate_{request.param}.mtp", mode=request.param, seed=11,
                           additive=[1.0, 0.7])


def test_reader_gate_fields(gate_model):
    m = load_mtp(gate_model)
    g = m.gate
    assert g is not None and g["nbody"] == m.sh_k_max
    assert len(m.scalar_body) == m.alpha_scalar_moments
    assert sorted(set(g["body_of"])) == list(range(g["nbody"]))
    assert all(m.alpha_moment_mapping[q] == mo for q, mo in zip(g["scalar_indices"], g["moment_of"]))


def _mutate(path, tmp_path, name, old, new, count=1):
    text = open(path).read()
    assert old in text, old
    p = tmp_path / name
    p.write_text(text.replace(old, new, count))
    return str(p)


CASES = [
    ("two_layer_gate_mode = mu-scalar-full", "two_layer_gate_mode = legacy", "legacy gate models"),
    ("two_layer_gate_mode = mu-scalar-full", "two_layer_gate_mode = fancy", "Unsupported SUS2_SH two_layer_gate_mode"),
    ("two_layer_gate_site_mode = neighbor", "two_layer_gate_site_mode = double", "Double-site gate"),
    ("two_layer_gate_radial_mode = shared-radial", "two_layer_gate_radial_mode = own", "shared-radial"),
    ("two_layer_gate_tanh_amplitude = 0.5", "two_layer_gate_tanh_amplitude = 1.5", "amplitude"),
    ("two_layer_gate_body_order_max = 4", "two_layer_gate_body_order_max = 5", "sh_k_max + 1"),
    ("two_layer_gate_radial_coeff_count = 96", "two_layer_gate_radial_coeff_count = 95", "radial coefficient count"),
    ("two_layer_gate_enabled = 1", "two_layer_gate_enabled = 1\ntwo_layer_gate_bias = 0", "two_layer_gate_bias"),
    ("two_layer_gate_enabled = 1", "two_layer_gate_enabled = 1\ntwo_layer_gate_body_mix_weight_count = 3",
     "should not contain body-mix"),
    ("two_layer_gate_enabled = 1", "two_layer_gate_enabled = 1\ntwo_layer_gate_additive_coeff_count = 3",
     "additive coefficient count"),
]


@pytest.mark.parametrize("old,new,msg", CASES)
def test_gate_errors_match_reference(l3k3_path, model_dir, tmp_path, old, new, msg):
    path = models.add_gate(l3k3_path, f"{model_dir}/gate_err_base.mtp", mode="mu-scalar-full", seed=12)
    bad = _mutate(path, tmp_path, "bad.mtp", old, new)
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.sus2sh_create(bad.encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert msg in lib.sus2sh_last_error().decode()
    with pytest.raises(MtpError, match=re.escape(msg)):
        load_mtp(bad)


def test_gate_needs_scalar_info_and_buckets(l3k3_path, model_dir, tmp_path):
    path = models.add_gate(l3k3_path, f"{model_dir}/gate_err_base2.mtp", mode="mu-body-linear-combo", seed=13)
    text = open(path).read()
    bad = tmp_path / "noinfo.mtp"
    bad.write_text(re.sub(r"sh_scalar_info_count = \d+\nsh_scalar_info = \{.*\}\n", "", text))
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.sus2sh_create(str(bad).encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "requires sh_scalar_info" in lib.sus2sh_last_error().decode()
    with pytest.raises(MtpError, match="requires sh_scalar_info"):
        load_mtp(str(bad))
    # keep only body-order-2 signals: the body-3 and body-4 buckets are missing
    m = load_mtp(path)
    two = [q for q in m.gate["scalar_indices"] if m.scalar_body[q] == 2]
    t2 = re.sub(r"two_layer_gate_weight_count = \d+", f"two_layer_gate_weight_count = {len(two)}", text)
    t2 = re.sub(r"two_layer_gate_scalar_indices = \{[^}]*\}",
                "two_layer_gate_scalar_indices = {" + ", ".join(map(str, two)) + "}", t2)
    t2 = re.sub(r"two_layer_gate_weights = \{[^}]*\}",
                "two_layer_gate_weights = {" + ", ".join(["0.001"] * len(two)) + "}", t2)
    bad2 = tmp_path / "buckets.mtp"
    bad2.write_text(t2)
    assert lib.sus2sh_create(str(bad2).encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "misses a required body-order bucket" in lib.sus2sh_last_error().decode()
    with pytest.raises(MtpError, match="misses a required body-order bucket"):
        load_mtp(str(bad2))


def test_oracle_gate_forces_and_virial(gate_model):
    orc = O.Oracle(gate_model)
    box, types, pos = structures.fcc(2, 2, 2, 3.8, (0.5, 0.5), 0.12, seed=14)
    pe, f, v = orc.efs(box.cpu_h, box.pbc, types, pos)
    hstep = 1e-5
    rng = np.random.default_rng(3)
    for i in rng.choice(types.size, 4, replace=False):
        for a in range(3):
            p1 = pos.copy(); p1[a, i] += hstep
            p2 = pos.copy(); p2[a, i] -= hstep
            fd = -(orc.efs(box.cpu_h, box.pbc, types, p1)[0].sum()
                   - orc.efs(box.cpu_h, box.pbc, types, p2)[0].sum()) / (2 * hstep)
            assert abs(fd - f[a, i]) < 1e-7 * max(1.0, abs(f[a, i]))
    H = box.cpu_h.reshape(3, 3)
    for a, b, q in ((0, 0, 0), (1, 2, 5), (2, 1, 8)):
        E = []
        for sgn in (1, -1):
            D = np.eye(3)
            D[a, b] += sgn * hstep
            E.append(orc.efs((D @ H).ravel(), box.pbc, types, D @ pos)[0].sum())
        assert abs(-(E[0] - E[1]) / (2 * hstep) - v[q].sum()) < 1e-6 * max(1.0, abs(v[q].sum()))
