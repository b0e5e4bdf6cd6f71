"""The .mtp reader never crashes on a damaged file.

GPUMD's `potential` command loads the model inside the MD program, so a reader
that crashed (a read out of bounds, an unchecked count driving an allocation or
an index) would take the whole run down.  Every truncated or corrupted copy of a
valid model must come back from sus2sh_create as an error code with a message:
SUS2SH_E_INPUT for a file the reader rejects, or, for a mutation that leaves a
readable model, whatever the CUDA set-up returns (the child process sees no
GPU).  The calls run in a child process so that a crash fails the test instead
of ending the test run.
"""
import json
import os
import re
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, sys
sys.path.insert(0, sys.argv[1])
from sus2sh import _lib
lib = _lib.load()
for path in sys.argv[2:]:
    h = ctypes.c_void_p()
    rc = lib.sus2sh_create(path.encode(), 0, 0, None, ctypes.byref(h))
    if rc == 0:
        lib.sus2sh_destroy(h)
    print(json.dumps([path, rc, lib.sus2sh_last_error().decode(errors="replace")]), flush=True)
"""

COUNT_KEYS = ["species_count", "sh_l_max", "sh_k_max", "sh_body_order", "radial_basis_size", "radial_funcs_count",
              "alpha_moments_count", "alpha_index_basic_count", "sh_product_count", "alpha_scalar_moments",
              "sh_scalar_info_count", "max_dist", "scaling"]
BAD_NUMBERS = ["", "abc", "nan", "inf", "-1", "0", "1", "2147483648", "99999999", "1e308", "3.5", "0x10"]


def mutations(text):
    """(name, text) pairs: truncations, corrupted counts and lists, indices out of range."""
    out = []
    n = len(text)
    for k in range(1, 80):
        out.append((f"trunc{k}", text[: n * k // 80]))
    for m in re.finditer(r"^\s*([a-z_]+)\s*=", text, flags=re.M):
        out.append((f"cut_after_{m.group(1)}", text[: m.end()]))
    for key in COUNT_KEYS:
        m = re.search(r"^(\s*" + key + r" = )(\S+)$", text, flags=re.M)
        assert m, key
        for bad in BAD_NUMBERS:
            out.append((f"{key}={bad}", text[: m.start(2)] + bad + text[m.end(2):]))
    # brace lists: unclosed, a garbage element, an element too many or too few
    for key in ["shift_coeffs", "scal_coeffs", "alpha_index_basic", "sh_products", "alpha_moment_mapping",
                "sh_scalar_info", "species_coeffs", "moment_coeffs"]:
        m = re.search(r"^" + key + r" = \{(.*)\}$", text, flags=re.M)
        assert m, key
        body = m.group(1)
        for tag, nb in [("unclosed", body + "\n"), ("garbage", "zz, " + body), ("extra", body + ", 1"),
                        ("short", body.rsplit(",", 1)[0]), ("empty", "")]:
            repl = (key + " = {" + nb) if tag == "unclosed" else (key + " = {" + nb + "}")
            out.append((f"{key}_{tag}", text[: m.start()] + repl + text[m.end():]))
    # indices out of range: products, basic-moment triples, the scalar mapping
    prod = re.search(r"sh_products = \{\{(\d+), (\d+), (\d+),", text)
    for tag, (a, b, c) in {"left": (99999, 1, 48), "right": (0, -5, 48), "target": (0, 0, 2**31 - 1),
                           "target_neg": (0, 0, -1)}.items():
        out.append((f"product_{tag}", text.replace(prod.group(0), f"sh_products = {{{{{a}, {b}, {c},", 1)))
    basic = re.search(r"alpha_index_basic = \{\{(-?\d+), (-?\d+), (-?\d+)\}", text)
    for tag, (k, l, mm) in {"k": (9, 3, 0), "l": (0, 9, 0), "m": (0, 1, 5), "neg": (-1, 0, 0)}.items():
        out.append((f"basic_{tag}", text.replace(basic.group(0), f"alpha_index_basic = {{{{{k}, {l}, {mm}}}", 1)))
    amap = re.search(r"alpha_moment_mapping = \{(\d+)", text)
    for tag, v in {"big": 99999, "neg": -1, "huge": 2**40}.items():
        out.append((f"mapping_{tag}", text.replace(amap.group(0), f"alpha_moment_mapping = {{{v}", 1)))
    out.append(("radial_group_long", text.replace("\tradial_coeffs\n\t\t{", "\tradial_coeffs\n\t\t{1e300, ", 1)))
    out.append(("radial_group_short", re.sub(r"(\tradial_coeffs\n\t\t\{)[^,]+, ", r"\1", text, count=1)))
    out.append(("binary_noise", text[: n // 2] + "\x00\xff\x01garbage\x00" + text[n // 2:]))
    return out


def test_damaged_models_return_error_codes(l3k3_path, tmp_path):
    text = open(l3k3_path).read()
    cases = mutations(text)
    paths = []
    for i, (name, body) in enumerate(cases):
        p = tmp_path / f"m{i:03d}.mtp"
        p.write_text(body, errors="surrogateescape")
        paths.append(str(p))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    proc = subprocess.run([sys.executable, "-c", CHILD, os.path.join(REPO, "gpumd-sus2-sh_b200")] + paths, env=env,
                          capture_output=True, text=True, timeout=600)
    seen = [json.loads(line) for line in proc.stdout.splitlines() if line.startswith("[")]
    if proc.returncode != 0:
        last = cases[len(seen)][0] if len(seen) < len(cases) else "?"
        raise AssertionError(f"reader crashed (exit {proc.returncode}) on mutation {last!r}: {proc.stderr[-500:]}")
    assert len(seen) == len(cases)
    names = {p: name for p, (name, _) in zip(paths, cases)}
    rejected = 0
    for path, rc, msg in seen:
        assert rc in (-1, -2, -3), (names[path], rc, msg)
        assert msg, names[path]
        rejected += rc == -1
    # nearly every mutation is a malformed model
    assert rejected > 0.8 * len(cases)
