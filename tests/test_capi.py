"""CPU checks of the C-ABI library: it loads, exports every symbol the public
headers declare, and reports malformed models as input errors (the reference
prints and exits, src/force/sus2_sh.cu:269-273) without touching a GPU."""
import ctypes
import os
import re

import pytest

import sus2sh
from sus2sh import _lib

INCLUDE = os.path.join(os.path.dirname(__file__), "..", "include")


def declared_functions(*headers):
    names = set()
    for h in headers:
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(sus2sh_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    decl = declared_functions("sus2sh.h", "sus2sh_diag.h")
    assert decl == set(_lib.EXPORTS)
    for name in decl:
        assert hasattr(lib, name), name


def test_tools_library_is_separate_from_the_engine():
    """The writer, integrator, insertion and FMA probe are in
    libsus2sh_tools.so, and libsus2sh.so exports none of them."""
    import subprocess
    tools = _lib.load_tools()
    decl = declared_functions("sus2sh_tools.h")
    assert decl == set(_lib.TOOLS_EXPORTS)
    for name in decl:
        assert hasattr(tools, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], stdout=subprocess.PIPE, text=True).stdout
    engine_syms = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert not (decl & engine_syms), decl & engine_syms


def test_is_sus2_sh_file(l3k3_path, tmp_path):
    assert sus2sh.is_sus2_sh_potential_file(l3k3_path)
    p = tmp_path / "plain.mtp"
    p.write_text("MTP\nversion = 1.1.0\npotential_tag = \n")
    assert not sus2sh.is_sus2_sh_potential_file(str(p))
    assert not sus2sh.is_sus2_sh_potential_file(str(tmp_path / "missing.mtp"))


def _mutate(src, dst, old, new, count=1):
    text = open(src).read()
    assert old in text, old
    open(dst, "w").write(text.replace(old, new, count))
    return str(dst)


CASES = [
    ("version = 1.1.0", "version = 1.0.0", "supports only version = 1.1.0"),
    ("potential_tag = SUS2-SH", "potential_tag = SUS2", "non-SUS2-SH"),
    ("scaling_map = LK", "scaling_map = L", "scaling_map = LK"),
    ("sh_body_order = 4", "sh_body_order = 7", "sh_body_order in [2,6]"),
    ("radial_basis_type = RBChebyshev_sss", "radial_basis_type = RBShapeev", "Unsupported SUS2_SH radial_basis_type"),
    ("radial_funcs_count = 12", "radial_funcs_count = 11", "inconsistent sh_k_max/radial_funcs_count"),
    ("alpha_index_basic_count = 48", "alpha_index_basic_count = 47", "alpha_index_basic size"),
    ("sh_product_count = 806", "sh_product_count = 805", "sh_products size"),
    ("sh_parity = even", "sh_parity = odd", "even parity"),
    # sh_scalar_info is checked before the coefficient dimensions (sus2_sh.cu:2354-2410)
    ("alpha_scalar_moments = 107", "alpha_scalar_moments = 106", "sh_scalar_info_count should equal"),
    ("sh_scalar_info_count = 107", "sh_scalar_info_count = 106", "sh_scalar_info_count should equal"),
    ("shift_coeffs = {-3.5, ", "shift_coeffs = {", "coefficient dimensions"),
]


@pytest.mark.parametrize("old,new,msg", CASES)
def test_malformed_model_is_input_error(l3k3_path, tmp_path, old, new, msg):
    bad = _mutate(l3k3_path, tmp_path / "bad.mtp", old, new)
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.sus2sh_create(bad.encode(), 0, 0, None, ctypes.byref(h))
    assert rc == -1
    assert msg in lib.sus2sh_last_error().decode()
    # the oracle reader rejects the same file
    from sus2sh_graph import MtpError, load_mtp
    with pytest.raises(MtpError):
        load_mtp(bad)


def test_missing_token_and_bad_products(l3k3_path, tmp_path):
    lib = _lib.load()
    h = ctypes.c_void_p()
    bad = _mutate(l3k3_path, tmp_path / "nomax.mtp", "max_dist =", "maximum =")
    assert lib.sus2sh_create(bad.encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "Missing token" in lib.sus2sh_last_error().decode()
    # a product writing into a basic moment
    text = open(l3k3_path).read()
    m = re.search(r"sh_products = \{\{(\d+), (\d+), (\d+),", text)
    t2 = text.replace(m.group(0), f"sh_products = {{{{{m.group(1)}, {m.group(2)}, 0,", 1)
    p = tmp_path / "basicwrite.mtp"
    p.write_text(t2)
    assert lib.sus2sh_create(str(p).encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "writes into a basic moment" in lib.sus2sh_last_error().decode()
    assert lib.sus2sh_create(str(tmp_path / "none.mtp").encode(), 0, 0, None, ctypes.byref(h)) == -1
    assert "Failed to open" in lib.sus2sh_last_error().decode()


def test_bad_options(l3k3_path):
    lib = _lib.load()
    h = ctypes.c_void_p()
    opts = (ctypes.c_char_p * 3)(b"Cu", b"Zr", b"sus2_float=maybe")
    rc = lib.sus2sh_create(l3k3_path.encode(), 0, 3, ctypes.cast(opts, ctypes.c_void_p), ctypes.byref(h))
    assert rc == -1 and "Invalid boolean" in lib.sus2sh_last_error().decode()
    opts = (ctypes.c_char_p * 3)(b"Cu", b"Zr", b"sus2_radial_direct=0")
    rc = lib.sus2sh_create(l3k3_path.encode(), 0, 3, ctypes.cast(opts, ctypes.c_void_p), ctypes.byref(h))
    assert rc == -1 and "direct radial" in lib.sus2sh_last_error().decode()


def test_null_arguments_rejected():
    lib = _lib.load()
    assert lib.sus2sh_create(None, 0, 0, None, None) == -3
    assert lib.sus2sh_compute(None, 10, None, None, None, None, None, None, None, None) == -3
    assert lib.sus2sh_sync(None, None) == -3


def test_model_fixture_matches_the_writer(tmp_path):
    """tests/golden/models/l3k3.mtp (read by the benchmark's reference arm)
    is exactly what the seeded writer produces for preset l3k3."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_model_fixtures as fx
    fresh = fx.write_fresh("l3k3", str(tmp_path))
    assert open(fresh, "rb").read() == open(fx.FIXTURES["l3k3"], "rb").read()
