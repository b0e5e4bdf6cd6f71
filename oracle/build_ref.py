"""Test infrastructure only: compiles the parts of the reference that build
from their own few source files, straight from the reference tree, into
``oracle/_ref/`` (git-ignored).

* ``libref_zbl.so``  -- ``oracle/ref_zbl_harness.cpp`` around the reference's
  ZBL header ``src/force/sus2_zbl_common.cuh`` (header-only, plain C++ when
  ``__CUDACC__`` is undefined).
* ``zbl_common_check`` -- the reference's own unit test
  ``codex_tests/gpumd_sh_zbl_common_check.cpp``, unmodified.

The SUS2-SH engine itself (``src/force/sus2_sh.cu``) needs the GPUMD tree,
nvcc and its CUDA kernels and is not built here; the graph and energy oracle
is pinned by the reference's published known-answer data instead.
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
    return {k: p for k, p in (("zbl_lib", LIB_ZBL), ("zbl_check", BIN_ZBL_CHECK)) if os.path.exists(p)}


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else REF_ROOT, force=True))
