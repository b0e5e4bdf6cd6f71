"""The engine's model reader accepts and rejects what the reference's does.

The reference's constructor (``SUS2_SH::SUS2_SH``, ``src/force/sus2_sh.cu``:
``load_sh_model`` :2105-2482, option parsing, standard-graph match and graph
metadata) runs unmodified from ``oracle/_ref/ref_sus2sh load`` (built by
``oracle/build_ref.py`` against minimal GPUMD stand-ins; host memory, no
GPU).  Every model here goes through it and through ``sus2sh_create``:

* a file the reference rejects with a message (its ``exit(1)``) is rejected
  by the engine with the same message (SUS2SH_E_INPUT);
* a file the reference accepts is accepted by the engine's reader (on a
  machine without a GPU ``sus2sh_create`` then fails in its CUDA set-up, not
  with SUS2SH_E_INPUT);
* a file on which the reference dies (an uncaught ``std::stoi``/``std::stod``
  exception: empty or non-numeric counts) gets an input error from the engine.

Deliberate differences, each listed here and nowhere else accepted:
``max_dist`` must be positive (the reference runs with a non-positive
cutoff); ``species_count`` must lie in [1, 16] (checked before the reference's
own row-size check fires); the unsupported-radial-basis message lists the
engine's own set of radial maps.
"""
import json
import os
import subprocess
import sys

import pytest

import ref_engine
import test_mtp_fuzz as fuzz

pytestmark = pytest.mark.skipif(not ref_engine.available(), reason="oracle/_ref/ref_sus2sh not built")

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
E_INPUT = -1

# (mutation name -> the engine's message) where the engine deliberately differs
ENGINE_ONLY_REJECTS = {
    "max_dist=nan": "SUS2_SH max_dist must be positive.",
    "max_dist=-1": "SUS2_SH max_dist must be positive.",
    "max_dist=0": "SUS2_SH max_dist must be positive.",
}
OTHER_MESSAGE = {
    "species_count=0": "SUS2_SH engine supports species_count in [1,16].",
    "species_count=99999999": "SUS2_SH engine supports species_count in [1,16].",
    "species_count=0x10": "SUS2_SH engine supports species_count in [1,16].",
}


def _engine_create(paths, opts_per_path):
    """sus2sh_create on each file in one child process: [(rc, message)]."""
    child = r"""
import ctypes, json, sys
sys.path.insert(0, sys.argv[1])
from sus2sh import _lib
lib = _lib.load()
jobs = json.loads(sys.stdin.read())
for path, opts in jobs:
    arr = (ctypes.c_char_p * max(1, len(opts)))(*[o.encode() for o in opts])
    h = ctypes.c_void_p()
    rc = lib.sus2sh_create(path.encode(), 0, len(opts), arr if opts else None, ctypes.byref(h))
    if rc == 0:
        lib.sus2sh_destroy(h)
    print(json.dumps([rc, lib.sus2sh_last_error().decode(errors="replace")]), flush=True)
"""
    env = {k: v for k, v in os.environ.items() if not k.startswith("SUS2_")}
    env["CUDA_VISIBLE_DEVICES"] = env.get("CUDA_VISIBLE_DEVICES", "")
    p = subprocess.run([sys.executable, "-c", child, os.path.join(REPO, "gpumd-sus2-sh_b200")],
                       input=json.dumps([[a, list(b)] for a, b in zip(paths, opts_per_path)]),
                       stdout=subprocess.PIPE, text=True, timeout=1200, env=env)
    assert p.returncode == 0, p.stdout[-2000:]
    out = [json.loads(ln) for ln in p.stdout.splitlines() if ln.startswith("[")]
    assert len(out) == len(paths)
    return out


def _check(name, ref, rc, msg):
    if name in ENGINE_ONLY_REJECTS:
        assert ref.accepted, (name, ref.message)
        assert rc == E_INPUT and msg == ENGINE_ONLY_REJECTS[name], (name, rc, msg)
        return "engine_only"
    if ref.crashed:
        assert rc == E_INPUT and msg, (name, rc, msg)
        return "reference_crash"
    if ref.accepted:
        assert rc != E_INPUT, (name, rc, msg)
        return "both_accept"
    assert rc == E_INPUT, (name, rc, msg, ref.message)
    if name in OTHER_MESSAGE:
        assert msg == OTHER_MESSAGE[name], (name, msg)
    elif ref.message.startswith("Unsupported SUS2_SH radial_basis_type in GPUMD:"):
        assert msg.startswith("Unsupported SUS2_SH radial_basis_type:"), (name, msg)
    else:
        assert msg == ref.message, (name, msg, ref.message)
    return "both_reject"


def test_damaged_models_same_verdict_as_reference(l3k3_path, tmp_path):
    text = open(l3k3_path).read()
    names, paths = [], []
    for name, t in fuzz.mutations(text):
        p = tmp_path / (name.replace("/", "_") + ".mtp")
        p.write_text(t, errors="surrogateescape")
        names.append(name)
        paths.append(str(p))
    ours = _engine_create(paths, [("Cu", "Zr")] * len(paths))
    counts = {}
    for name, path, (rc, msg) in zip(names, paths, ours):
        kind = _check(name, ref_engine.load(path, ("Cu", "Zr")), rc, msg)
        counts[kind] = counts.get(kind, 0) + 1
    # the corpus exercises every branch
    assert counts.get("both_reject", 0) > 200 and counts.get("both_accept", 0) > 10, counts
    assert counts.get("reference_crash", 0) > 0 and counts.get("engine_only", 0) == 3, counts


def _variants(l3k3_path, d):
    from sus2sh import models
    out = [("l3k3", l3k3_path, ("Cu", "Zr"))]
    z = models.add_zbl(l3k3_path, os.path.join(d, "zbl.mtp"))
    out.append(("zbl", z, ("Cu", "Zr")))
    out.append(("zbl_no_symbols", z, ()))
    for mode in ("mu-scalar-full", "mu-body-linear-combo"):
        out.append((f"gate_{mode}", models.add_gate(l3k3_path, os.path.join(d, f"gate_{mode}.mtp"), mode=mode),
                    ("Cu", "Zr")))
    for L, K, body in ((1, 1, 3), (2, 2, 4), (5, 2, 3), (6, 1, 3)):
        p = models.write_model(os.path.join(d, f"l{L}k{K}b{body}.mtp"), l_max=L, k_max=K, body_order=body, seed=L)
        out.append((f"l{L}k{K}b{body}", p, ("Cu", "Zr")))
    # options: precision switches, the reference's accepted tuning tokens, and
    # the direct-radial switch the reference rejects
    for opts in (("sus2_float=0",), ("sus2_sh_float=1",), ("sus2_float=maybe",), ("sus2_radial_direct=0",),
                 ("sus2_sh_profile=1", "sus2_sh_profile_interval=7"), ("sus2_factor_pruning=q-total",),
                 ("sus2_factor_pruning=bogus",)):
        out.append(("opts_" + "_".join(opts), l3k3_path, ("Cu", "Zr", *opts)))
    return out


def test_model_variants_and_options_same_verdict_as_reference(l3k3_path, tmp_path):
    cases = _variants(l3k3_path, str(tmp_path))
    ours = _engine_create([p for _, p, _ in cases], [o for _, _, o in cases])
    verdicts = {}
    for (name, path, opts), (rc, msg) in zip(cases, ours):
        ref = ref_engine.load(path, opts)
        verdicts[name] = _check(name, ref, rc, msg)
    assert verdicts["l3k3"] == "both_accept" and verdicts["zbl"] == "both_accept"
    assert verdicts["opts_sus2_radial_direct=0"] == "both_reject"
    assert verdicts["opts_sus2_float=maybe"] == "both_reject"
