"""Test infrastructure only: runs the reference's own SUS2-SH engine.

``oracle/_ref/ref_sus2sh`` is the reference's ``src/force/sus2_sh.cu``,
unmodified, compiled for sm_100a against minimal GPUMD stand-ins
(``oracle/gpumd_stub/``) by ``oracle/build_ref.py``.  This module drives it as
a child process, so the reference's ``exit(1)`` on input errors
(``sus2_sh.cu:269-273``) and its CUDA context stay out of the caller's
process:

* ``load(path, opts)``: the reference's constructor (model reader, standard
  graph match, graph metadata) in host memory, no GPU needed;
* ``run(path, box_h, pbc, types, pos, opts, steps, warmup)``: energies, forces
  and virials from ``SUS2_SH::compute`` on a GPU, called as GPUMD's
  ``Force::compute`` calls it (outputs zeroed first), plus the mean
  CUDA-event time of one call.

Only the tests and the benchmark's reference arm use it.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "ref_sus2sh")


def available() -> bool:
    return os.path.exists(BIN) and os.access(BIN, os.X_OK)


class LoadResult:
    """Outcome of the reference's constructor on one model file."""

    def __init__(self, returncode: int, stdout: str):
        self.returncode = returncode
        self.stdout = stdout
        self.accepted = returncode == 0 and "SUS2SH_REF_LOADED" in stdout
        lines = [ln for ln in stdout.splitlines() if ln.strip()]
        # an input error is the last line the reference prints before exit(1)
        self.message = "" if self.accepted or not lines else lines[-1].strip()
        self.crashed = returncode < 0 or returncode > 1


def load(path: str, opts=(), timeout: float = 120.0) -> LoadResult:
    env = {k: v for k, v in os.environ.items() if not k.startswith("SUS2_")}
    p = subprocess.run([BIN, "load", path, *opts], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       timeout=timeout, env=env)
    return LoadResult(p.returncode, p.stdout.decode(errors="replace"))


def write_input(fname: str, box_h, pbc, types, pos) -> None:
    """The driver's binary input: int32 N, pbc[3], double h[9], int32
    type[N], double position[3N] (SoA)."""
    types = np.ascontiguousarray(types, dtype=np.int32)
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(3, -1)
    N = types.size
    with open(fname, "wb") as f:
        np.asarray([N], dtype=np.int32).tofile(f)
        np.asarray(pbc, dtype=np.int32).reshape(3).tofile(f)
        np.asarray(box_h, dtype=np.float64).reshape(9).tofile(f)
        types.tofile(f)
        pos.tofile(f)


def run(path: str, box_h, pbc, types, pos, opts=(), steps: int = 1, warmup: int = 0, timeout: float = 600.0):
    """Returns (potential[N], force[3, N], virial[9, N], ms_per_call, stdout).
    ``opts`` are the run.in tokens after the file name (species symbols
    first).  Raises RuntimeError when the reference exits non-zero."""
    N = int(np.asarray(types).size)
    env = {k: v for k, v in os.environ.items() if not k.startswith("SUS2_")}
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        write_input(fin, box_h, pbc, types, pos)
        p = subprocess.run([BIN, "run", path, fin, fout, str(steps), str(warmup), *opts], stdout=subprocess.PIPE,
                           stderr=subprocess.STDOUT, timeout=timeout, env=env)
        out = p.stdout.decode(errors="replace")
        if p.returncode != 0:
            raise RuntimeError(f"reference engine exited with {p.returncode}: {out[-2000:]}")
        data = np.fromfile(fout, dtype=np.float64)
    if data.size != 13 * N:
        raise RuntimeError(f"reference engine wrote {data.size} values, expected {13 * N}")
    pe = data[:N]
    f = data[N:4 * N].reshape(3, N)
    w = data[4 * N:].reshape(9, N)
    ms = timing(out).get("ref_ms_per_step", float("nan"))
    return pe, f, w, ms, out


def timing(stdout: str) -> dict:
    """The driver's timing line: mean, median, min and max ms per call."""
    line = [ln for ln in stdout.splitlines() if ln.startswith('{"ref_ms_per_step"')]
    return json.loads(line[-1]) if line else {}


def profile_stages(stdout: str) -> dict | None:
    """The reference's own stage profile line (option sus2_sh_profile=1,
    printed every sus2_sh_profile_interval calls, sus2_sh.cu:10638-10660):
    the last one, as {stage: ms per call}."""
    last = None
    for ln in stdout.splitlines():
        if ln.startswith("SUS2-SH profile avg over"):
            last = ln
    if last is None:
        return None
    out = {}
    for part in last.split(":", 1)[1].split(","):
        if "=" in part:
            k, v = part.split("=", 1)
            out[k.strip()] = float(v.strip().split()[0])
    return out


if __name__ == "__main__":
    # python oracle/ref_engine.py frame <out.bin>: the benchmark's static
    # 1,024,000-atom Cu-Zr frame (80x80x40 FCC, a = 3.8 A, 64/36, seed 1000)
    # as input for oracle/_ref/ref_sus2sh run, e.g. to profile the reference.
    import sys
    if len(sys.argv) != 3 or sys.argv[1] != "frame":
        raise SystemExit("usage: ref_engine.py frame <out.bin>")
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "gpumd-sus2-sh_b200"))
    from sus2sh import structures
    box, types, pos = structures.fcc(80, 80, 40, 3.8, (0.64, 0.36), 0.0, seed=1000)
    write_input(sys.argv[2], box.cpu_h, box.pbc, types, pos)
    print(f"wrote {types.size} atoms to {sys.argv[2]}")
