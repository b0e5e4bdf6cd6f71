"""Test infrastructure only: compiles the parts of the reference that build
from their own few source files, straight from the reference tree, into
``oracle/_ref/`` (git-ignored).

* ``libref_zbl.so``  -- ``oracle/ref_zbl_harness.cpp`` around the reference's
  ZBL header ``src/force/sus2_zbl_common.cuh`` (header-only, plain C++ when
  ``__CUDACC__`` is undefined).
* ``zbl_common_check`` -- the reference's own unit test
  ``codex_tests/gpumd_sh_zbl_common_check.cpp``, unmodified.
* ``ref_sus2sh`` -- the reference's SUS2-SH engine ``src/force/sus2_sh.cu``,
  unmodified, compiled with nvcc for sm_100a against the minimal GPUMD
  stand-ins in ``oracle/gpumd_stub/`` (box, device array, error macros,
  potential base class, neighbour search) and linked with the command-line
  driver ``oracle/ref_sus2sh_main.cu``.  ``ref_sus2sh load`` runs the
  reference's model reader and graph set-up without a GPU; ``ref_sus2sh run``
  evaluates energies, forces and virials on a GPU.  The engine's translation
  unit takes several minutes to compile, so its object is kept and rebuilt
  only when a source it depends on changes.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# The reference checkout: $SUS2SH_REFERENCE_ROOT, else a directory named
# "reference" beside this repository's root; absent (the usual case away from
# the development machine) means the prebuilt files in _ref/ are used as they are.
REF_ROOT = os.environ.get("SUS2SH_REFERENCE_ROOT") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")

ZBL_HEADER = os.path.join("src", "force", "sus2_zbl_common.cuh")
ZBL_TEST = os.path.join("codex_tests", "gpumd_sh_zbl_common_check.cpp")
LIB_ZBL = os.path.join(OUT, "libref_zbl.so")
BIN_ZBL_CHECK = os.path.join(OUT, "zbl_common_check")

ENGINE_DIR = os.path.join("src", "force")
ENGINE_SRC = os.path.join(ENGINE_DIR, "sus2_sh.cu")
STUB = os.path.join(HERE, "gpumd_stub")
BIN_ENGINE = os.path.join(OUT, "ref_sus2sh")
NVCC = os.environ.get("NVCC", "nvcc")
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo"]


def _stale(target: str, sources) -> bool:
    return not os.path.exists(target) or os.path.getmtime(target) < max(os.path.getmtime(p) for p in sources)


def _stub_headers():
    out = []
    for d, _, files in os.walk(STUB):
        out += [os.path.join(d, f) for f in files if f.endswith(".cuh")]
    return out


def build_engine(root: str = REF_ROOT, force: bool = False) -> str | None:
    """Compiles the reference engine + stand-ins + driver into _ref/ref_sus2sh.
    Returns its path, or None when neither the reference tree nor a prebuilt
    binary is there."""
    if not reference_present(root) or not os.path.exists(os.path.join(root, ENGINE_SRC)):
        return BIN_ENGINE if os.path.exists(BIN_ENGINE) else None
    os.makedirs(OUT, exist_ok=True)
    fdir = os.path.join(root, ENGINE_DIR)
    inc = ["-I", STUB, "-I", fdir]
    engine_deps = [os.path.join(fdir, f) for f in ("sus2_sh.cu", "sus2_sh.cuh", "sus2_zbl_common.cuh")]
    objs = []
    for src, deps in ((os.path.join(root, ENGINE_SRC), engine_deps),
                      (os.path.join(STUB, "neighbor.cu"), []),
                      (os.path.join(HERE, "ref_sus2sh_main.cu"), [os.path.join(fdir, "sus2_sh.cuh")])):
        obj = os.path.join(OUT, os.path.splitext(os.path.basename(src))[0] + ".o")
        if force or _stale(obj, [src] + deps + _stub_headers()):
            subprocess.check_call([NVCC] + NVCC_FLAGS + inc + ["-c", "-o", obj, src])
        objs.append(obj)
    if force or _stale(BIN_ENGINE, objs):
        subprocess.check_call([NVCC] + NVCC_FLAGS + ["-o", BIN_ENGINE] + objs)
    return BIN_ENGINE


def reference_present(root: str = REF_ROOT) -> bool:
    return bool(root) and os.path.exists(os.path.join(root, ZBL_HEADER)) and os.path.exists(os.path.join(root, ZBL_TEST))


def build(root: str = REF_ROOT, force: bool = False) -> dict:
    """Builds both artefacts when the reference tree is present; returns the
    paths that exist afterwards (prebuilt files are kept when it is absent)."""
    if reference_present(root):
        os.makedirs(OUT, exist_ok=True)
        header = os.path.join(root, ZBL_HEADER)
        harness = os.path.join(HERE, "ref_zbl_harness.cpp")
        newest = max(os.path.getmtime(header), os.path.getmtime(harness))
        if force or not os.path.exists(LIB_ZBL) or os.path.getmtime(LIB_ZBL) < newest:
            subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", root, "-o", LIB_ZBL,
                                   harness])
        test_src = os.path.join(root, ZBL_TEST)
        if force or not os.path.exists(BIN_ZBL_CHECK) or os.path.getmtime(BIN_ZBL_CHECK) < max(
                os.path.getmtime(test_src), os.path.getmtime(header)):
            subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", root, "-o", BIN_ZBL_CHECK, test_src])
    build_engine(root, force)
    return {k: p for k, p in (("zbl_lib", LIB_ZBL), ("zbl_check", BIN_ZBL_CHECK), ("engine", BIN_ENGINE))
            if os.path.exists(p)}


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else REF_ROOT, force=True))
