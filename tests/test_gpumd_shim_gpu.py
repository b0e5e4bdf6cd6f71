"""The GPUMD shim, compiled and driven as GPUMD drives a potential.

``gpumd-sus2-sh_b200/gpumd/sus2_sh.cu`` is the drop-in for the reference's
``src/force/sus2_sh.cu`` (same class, constructor and compute signatures,
``src/force/sus2_sh.cuh:7-25``).  The test builds it with nvcc against the
GPUMD stand-ins of ``oracle/gpumd_stub`` and ``libsus2sh.so``, together with
``tests/gpumd_shim_driver.cu``, which zeroes the per-atom arrays and calls
``SUS2_SH::compute`` as ``Force::compute`` does (``src/force/force.cu:
513-519``).  The results must be the engine's (``sus2sh_compute`` through the
Python binding) and the oracle's; a compressed frame after a dilute one
overflows the neighbour list sized at the first step, and the shim's redo
branch must then give the full result.
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import sus2sh_oracle as O  # noqa: E402
from sus2sh import Box, structures  # noqa: E402
from test_parity_gpu import engine_efs  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gpumd-sus2-sh_b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "gpumd_shim_driver")
    nvcc = os.environ.get("NVCC", "nvcc")
    subprocess.check_call([nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-I", os.path.join(REPO, "oracle", "gpumd_stub"), "-I", os.path.join(REPO, "include"),
                           "-I", os.path.join(PKG, "gpumd"), "-o", out,
                           os.path.join(REPO, "tests", "gpumd_shim_driver.cu"),
                           os.path.join(PKG, "gpumd", "sus2_sh.cu"), "-L", PKG, "-lsus2sh",
                           "-Xlinker", "-rpath," + PKG])
    return out


def run_shim(driver, path, box, types, frames, opts=("Cu", "Zr")):
    N = types.size
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as fh:
            np.asarray([N], dtype=np.int32).tofile(fh)
            np.asarray(box.pbc, dtype=np.int32).tofile(fh)
            np.asarray(box.cpu_h, dtype=np.float64).tofile(fh)
            np.asarray(types, dtype=np.int32).tofile(fh)
            np.asarray([len(frames)], dtype=np.int32).tofile(fh)
            for p in frames:
                np.ascontiguousarray(p, dtype=np.float64).tofile(fh)
        p = subprocess.run([driver, path, fin, fout, *opts], stdout=subprocess.PIPE, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:]
        data = np.fromfile(fout, dtype=np.float64).reshape(len(frames), 13 * N)
    info = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    out = [(row[:N], row[N:4 * N].reshape(3, N), row[4 * N:].reshape(9, N)) for row in data]
    return out, info, p.stdout


@pytest.mark.parametrize("fp64", [False, True])
def test_shim_matches_engine_and_oracle(driver, l3k3_path, fp64):
    box, types, pos = structures.fcc(6, 6, 6, 3.8, (0.5, 0.5), 0.05, seed=61)
    opts = ("Cu", "Zr") + (("sus2_float=0",) if fp64 else ())
    rng = np.random.default_rng(1)
    frames = [pos, pos + rng.normal(0.0, 0.02, size=pos.shape)]
    out, info, _ = run_shim(driver, l3k3_path, box, types, frames, opts)
    assert info["recomputed_steps"] == 0 and info["rc"] == 5.0
    orc = O.Oracle(l3k3_path)
    for (pe, f, w), p in zip(out, frames):
        pe1, f1, w1 = engine_efs(l3k3_path, box, types, p, opts[2:])
        fbar = (1e-12 if fp64 else 1e-6) * max(1.0, np.abs(f1).max())
        assert np.abs(pe - pe1).max() < (1e-12 if fp64 else 1e-7) and np.abs(f - f1).max() < fbar
        assert np.abs(w - w1).max() < (1e-12 if fp64 else 1e-6) * max(1.0, np.abs(w1).max())
        pe0, f0, _ = orc.efs(box.cpu_h, box.pbc, types, p)
        assert np.abs(pe - pe0).max() < (1e-9 if fp64 else 1e-6)
        assert np.sqrt(((f - f0) ** 2).mean()) < (1e-9 if fp64 else 1e-5)


def test_shim_redoes_a_step_whose_rebuild_overflowed(driver, l3k3_path):
    # a dilute first frame sizes the list; a compressed cluster then
    # overflows it, and the shim recomputes that step with the grown list
    rng = np.random.default_rng(12)
    N = 200
    box = Box.orthorhombic(40.0, 40.0, 40.0)
    types = rng.integers(0, 2, N).astype(np.int32)
    dilute = rng.uniform(0, 40.0, size=(3, N))
    dense = 15.0 + rng.uniform(0, 9.0, size=(3, N))
    out, info, stdout = run_shim(driver, l3k3_path, box, types, [dilute, dense, dense])
    assert info["recomputed_steps"] == 1, stdout
    assert "step recomputed" in stdout
    pe0, f0, _ = O.Oracle(l3k3_path).efs(box.cpu_h, box.pbc, types, dense)
    for pe, f, _ in out[1:]:
        assert np.abs(pe - pe0).max() < 1e-4 * max(1.0, np.abs(pe0).max())
        assert np.sqrt(((f - f0) ** 2).mean()) < 1e-4 * max(1.0, np.sqrt((f0 ** 2).mean()))
