#!/usr/bin/env python
"""Benchmark of the SUS2-SH engine on the 1,024,000-atom Cu-Zr l3k3 NVE workload.

Workload (seeded synthetic stand-in for the reference's unshipped model.xyz and
p.mtp): FCC 80x80x40 cells, a = 3.8 A (1,024,000 atoms, box 304x304x152 A),
64/36 Cu/Zr random species, Maxwell-Boltzmann velocities at 200 K, NVE with
dt = 0.5 fs, Verlet skin 1.0 A and a forced neighbour rebuild every 10 steps.
Model: SUS2-SH l3k3 body 4 (L=3, K=3, Chebyshev-sss rb 8, rc 5.0 A, 248
moments, 806 CG products), random coefficients (radial ~N(0,0.1), moment
weights ~N(0,0.01)).

A step is one velocity-Verlet MD step (kick+drift, one energy/force/virial
evaluation through the C-ABI, kick) over all atoms of this rank.  The FP32
engine (sus2_float=1) is the headline; the plain FP64 engine (sus2_float=0)
runs the same workload for the FP32/FP64 ratio.  Multi-GPU runs are
independent replicas (weak scaling, no collective on the data path); timing is
the max over ranks.

--impl reference times the reference's own SUS2-SH engine: src/force/sus2_sh.cu,
unmodified, compiled for sm_100a against minimal GPUMD stand-ins
(oracle/_ref/ref_sus2sh, built by oracle/build_ref.py), on the same 1,024,000-atom
frame and model on this GPU, one SUS2_SH::compute per step (its default FP32
path; its FP64 path and its own stage profile are reported beside it).  Where
that build or a GPU is absent it falls back to the FP64 oracle port on this
host's cores.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "gpumd-sus2-sh_b200")
ORACLE = os.path.join(REPO, "oracle")
sys.path.insert(0, PKG)

METRIC = "atom-step/s, 1.024M-atom l3k3: FP32 vs FP64 path; force RMS err vs FP64 oracle"
CELLS = (80, 80, 40)
A = 3.8
DT = 0.5
TEMP = 200.0
SKIN = 1.0  # Verlet skin (A)
REBUILD = 10  # forced neighbour rebuild interval (steps)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, nargs=3, default=list(CELLS))
    ap.add_argument("--fp64-steps", type=int, default=-1,
                    help="timed steps of the FP64-engine leg (default: the same as --steps, so both legs "
                         "run under the same thermal and power conditions; 0 skips it)")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batch-cell and large-model fields")
    ap.add_argument("--large-only", type=int, default=0, metavar="ATOMS",
                    help="run only the large-model workload with this many atoms and print its fields "
                         "(profiling of the large-graph kernels)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def edges_within(box, pos, rc):
    """In-cutoff (directed) neighbour pairs of the structure, for the
    algorithmic flop count."""
    from scipy.spatial import cKDTree
    L = box.lengths()
    tree = cKDTree((pos.T % L), boxsize=L)
    counts = tree.query_ball_point(pos.T % L, r=rc * (1 - 1e-12), return_length=True)
    return int(counts.sum()) - pos.shape[1]  # minus self


# DRAM bytes of one k_force launch (dram__bytes_read.sum + dram__bytes_write.sum)
# from one ncu capture of the 524,288-atom l3k3 case (64x64x32 FCC cells, FP32,
# the build specialised to the model, 128-thread CTAs, walking the in-cutoff
# sub-list): 267.15 MB read + 39.17 MB written.  The traffic grows with the atom
# count, so the bench scales it per atom.
K_FORCE_DRAM_BYTES_PER_ATOM = (267.15e6 + 39.17e6) / 524288


def k_force_algorithmic_bytes(nbasic, cut_per_atom):
    """Bytes k_force must move per atom: adjoints G (4 nbasic), position and
    species (32), the in-cutoff neighbour count and list it walks (4 + 4 per
    pair inside rc), the FP32 scatter buffer (16) and the FP64 force (24,
    read + written) and virial (72, read + written) it accumulates into."""
    return 4 * nbasic + 32 + 4 + 4 * cut_per_atom + 16 + 2 * 24 + 2 * 72


def flops_model(kmu, rb, C, Bb, P):
    """Counting rule for algorithmic work (FMA = 2 flops)."""
    per_edge_basic = kmu * (2 * rb + 4) + 6 * C + 2 * Bb
    per_edge_force = kmu * (4 * rb + 6) + 20 * C + 8 * Bb + 24
    per_atom_product = 9 * P
    return per_edge_basic, per_edge_force, per_atom_product


def max_over_ranks(torch, values, world, device):
    """Each value's maximum over all ranks, by one MAX all-reduce: the slowest
    rank's time sets the whole job's throughput.  Every rank calls it at the
    same point of the run, so the ranks issue the same collectives in the same
    order."""
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.tolist()


def whole_job_rate(units_per_rank, world, steps, ms):
    """Units all ranks processed per second when the slowest rank took ms."""
    return units_per_rank * world * steps / (ms * 1e-3)


def fma_peak():
    """FP32 and FP64 FMA throughput of this GPU (libsus2sh_tools.so probe)."""
    from sus2sh import _lib
    lib = _lib.load_tools()
    v32, v64 = ctypes.c_double(0), ctypes.c_double(0)
    lib.sus2sh_measure_fma_peak(0, ctypes.byref(v32))
    lib.sus2sh_measure_fma_peak(1, ctypes.byref(v64))
    return v32.value, v64.value


def make_workload(model_dir, rank):
    from sus2sh import structures
    path = MODEL_FIXTURE  # the seeded l3k3 model (preset "l3k3"), shared with the reference arm
    box, types, pos = structures.fcc(*CELLS_RUN, A, (0.64, 0.36), 0.0, seed=1000 + rank)
    masses = [structures.AMU["Cu"], structures.AMU["Zr"]]
    vel = structures.maxwell_boltzmann(types, masses, TEMP, seed=2000 + rank)
    return path, box, types, pos, vel, masses


def run_md(torch, path, box, types, pos, vel, masses, steps, warmup, fp64, world, clocks=None):
    from sus2sh import SUS2_SH
    from sus2sh.md import NVE
    opts = ["Cu", "Zr", f"sus2_sh_skin={SKIN}", f"sus2_sh_rebuild_interval={REBUILD}"] + (["sus2_float=0"] if fp64 else [])
    pot = SUS2_SH(path, types.size, opts)
    md = NVE(pot, box, types, pos, vel, masses, dt_fs=DT)
    md.initial_force()
    for _ in range(warmup):
        md.step()
    torch.cuda.synchronize()
    if pot.sync() != 0:
        raise RuntimeError("neighbour list overflow during warm-up")
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    pot.profile(True)
    l0 = pot.info()["launches"]
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if clocks:
        clocks.start()
    t0 = time.time()
    s.record()
    for _ in range(steps):
        md.step()
    e.record()
    torch.cuda.synchronize()
    prof = pot.profile_read()
    info = pot.info()
    launches = info["launches"] - l0 + 2 * steps  # + kick_drift and kick
    flags = pot.sync()
    if flags:
        raise RuntimeError(f"neighbour list status {flags} during timed steps")
    timed_frame = md.pos.clone()  # the final frame of the timed steps (accuracy, CPU baseline, e2e)
    clk = None
    if clocks:
        # a timed region of a few tens of ms ends before nvidia-smi's first
        # samples; the same MD keeps the GPU under this load, untimed, until
        # the sampler has run for a second
        extra = 0
        while time.time() - t0 < 1.0:
            for _ in range(10):
                md.step()
            extra += 10
            pot.sync()  # a neighbour overflow here grows the list; the timed steps had none
        clk = clocks.stop()
        clk["window"] = (f"sampled from the start of the {steps} timed steps through {extra} further untimed "
                         "steps of the same MD (1 s in all)")
    if world > 1:
        torch.distributed.barrier()
    ms = s.elapsed_time(e)
    return pot, md, ms, prof, launches, clk, timed_frame


def force_error_vs_fp64(torch, path, box, types, x_dev):
    """FP32 and FP64 engines on the same frame: force RMS and max |dE|/atom,
    and the FP32 engine's (pe, f[3,N], w[9,N]) on host."""
    from sus2sh import SUS2_SH
    N = types.size
    dev = x_dev.device
    t = torch.as_tensor(types, device=dev)
    out = []
    for opt in ([], ["sus2_float=0"]):
        pot = SUS2_SH(path, N, ["Cu", "Zr"] + opt)
        pe = torch.zeros(N, dtype=torch.float64, device=dev)
        f = torch.zeros(3 * N, dtype=torch.float64, device=dev)
        w = torch.zeros(9 * N, dtype=torch.float64, device=dev)
        pot.compute(box, t, x_dev, pe, f, w)
        torch.cuda.synchronize()
        pot.sync()
        out.append((pe, f, w))
        pot.close()
    frms = float(torch.sqrt(((out[0][1] - out[1][1]) ** 2).mean()))
    de = float((out[0][0] - out[1][0]).abs().max())
    de_total = float((out[0][0].sum() - out[1][0].sum()).abs()) / N
    host32 = (out[0][0].cpu().numpy(), out[0][1].view(3, N).cpu().numpy(), out[0][2].view(9, N).cpu().numpy())
    return frms, de, de_total, host32


def e2e_run(torch, pot, box, types, x_dev, steps):
    """Host-buffer path: pinned host positions in, energies/forces out, every step."""
    N = types.size
    pin = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True)
    h_pos = pin(3 * N, torch.float64)
    h_pos.copy_(x_dev.cpu())
    h_type = pin(N, torch.int32)
    h_type.copy_(torch.as_tensor(types))
    h_pe = pin(N, torch.float64)
    h_f = pin(3 * N, torch.float64)
    h_vt = pin(9, torch.float64)
    for _ in range(2):
        pot.compute_host_ptrs(box, N, h_type.data_ptr(), h_pos.data_ptr(), h_pe.data_ptr(), h_f.data_ptr(),
                              h_vt.data_ptr())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        pot.compute_host_ptrs(box, N, h_type.data_ptr(), h_pos.data_ptr(), h_pe.data_ptr(), h_f.data_ptr(),
                              h_vt.data_ptr())
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return N * steps / dt, 28 * N, 32 * N + 72


def batch_cells_run(torch, path, ncells=4096, reps=10):
    """Uneven-cell batch workload: 4096 periodic random-insertion cells with
    16-512 atoms, density 0.06 A^-3, d_min 2.1 A, orthorhombic edge ratios
    0.8-1.25; energies, forces, virials and per-cell sums through one CUDA
    graph replay per evaluation (the stage kernels; the fused persistent
    kernel, option sus2_sh_batch_fused=1, timed beside them); then the
    batched parameter gradients."""
    from sus2sh import SUS2_SH, structures
    off, H, boxes, types, pos = structures.cell_batch(ncells, 16, 512, seed=4242)
    N = types.size
    dev = torch.device("cuda")
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    o = torch.as_tensor(off, device=dev)
    h = torch.as_tensor(H.reshape(-1).copy(), device=dev)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(opts):
        pot = SUS2_SH(path, N, ["Cu", "Zr"] + opts)
        pe, f, w, ce, cw = z(N), z(3 * N), z(9 * N), z(ncells), z(9 * ncells)
        pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce, cell_virial=cw)  # sizes lists, tunes tiles
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            pe.zero_(); f.zero_(); w.zero_()
            pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce, cell_virial=cw)
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            pe.zero_(); f.zero_(); w.zero_()
            pot.compute_batch(o, h, t, x, pe, f, w, cell_energy=ce, cell_virial=cw)
        for _ in range(3):
            g.replay()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        del g
        return pot, ms, pot.sync(), pot.info()

    fused, ms_fused, flags_fused, info_fused = timed(["sus2_sh_batch_fused=1"])
    fused.close()
    pot, ms, flags, info = timed([])
    nsc = info["scalars"]
    nrad = info["k_max"] * (info["l_max"] + 1) * info["rb_size"]
    ew = torch.ones(N, dtype=torch.float64, device=dev)
    fw = torch.full((3 * N,), 0.01, dtype=torch.float64, device=dev)
    gw, gc = z(nsc), z(nrad)
    pot.param_grad_batch(o, h, t, x, ew, fw, gw, gc)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(3):
        pot.param_grad_batch(o, h, t, x, ew, fw, gw, gc)
    e1.record()
    torch.cuda.synchronize()
    ms_grad = e0.elapsed_time(e1) / 3
    pot.close()
    return {"workload": "4096 uneven periodic cells (16-512 atoms), l3k3 FP32, one CUDA graph per evaluation",
            "cells": ncells, "atoms": N, "ms_per_eval": ms, "atom_evals_per_s": N / (ms * 1e-3),
            "evaluation": "stage kernels (geometry, pack, fill, moments, CG, forces, finalize, per-cell sums)",
            "fused_persistent_kernel": {
                "option": "sus2_sh_batch_fused=1", "ms_per_eval": ms_fused, "status_flags": flags_fused,
                "in_use": bool(info_fused["batch_fused"]), "registers": info_fused["batch_fused_registers"],
                "cta": info_fused["batch_fused_shape"] // 100, "min_ctas_per_sm": info_fused["batch_fused_shape"] % 100,
                "tile_atoms": info_fused["batch_fused_tile"]},
            "param_grad_ms": ms_grad, "status_flags": flags,
            "tiles": {"basic_block": info["basic_block"], "force_block": info["force_block"]}}


def large_model_run(torch, model_dir, reps=5, atoms=262144, opts=(), accuracy=True):
    """Large-model workload: Cu-Zr-Al body-5 L=4 K=4 rb10 rational-map model
    (5985 moments, 33,389 products) on 262,144 random-insertion atoms
    (0.06 A^-3, d_min 2.1 A, 50/35/15), FP32; static positions, one
    energy/force/virial evaluation per step."""
    from sus2sh import SUS2_SH, models, structures
    path = models.preset_model("l4k4", model_dir)
    box, types, pos = structures.random_insertion(atoms, 0.06, 2.1, (1.0, 1.0, 1.0), (0.5, 0.35, 0.15), seed=77)
    N = types.size
    dev = torch.device("cuda")
    pot = SUS2_SH(path, N, ["Cu", "Zr", "Al", *opts])
    t = torch.as_tensor(types, device=dev)
    x = torch.as_tensor(pos.reshape(-1).copy(), device=dev)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)
    pe, f, w = z(N), z(3 * N), z(9 * N)
    for _ in range(2):
        pot.compute(box, t, x, pe, f, w)
    torch.cuda.synchronize()
    pot.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        pot.compute(box, t, x, pe, f, w)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    prof = pot.profile_read()
    flags = pot.sync()
    info = pot.info()
    if accuracy:
        pe.zero_(); f.zero_(); w.zero_()
        pot.compute(box, t, x, pe, f, w)
        torch.cuda.synchronize()
    pot.close()
    out = {"workload": f"{N:,}-atom Cu-Zr-Al l4k4 body-5 rational model, FP32", "atoms": N,
           "cg_kernel": {0: "row interpreter", 1: "straight-line", 2: "component-split"}.get(info["cg_kind"]),
           "cg_build": {0: None, 1: "one NVRTC program", 2: "parallel relocatable units"}.get(info["cg_build"]),
           "cg_compile_ms": info["cg_jit_compile_ms"], "cg_from_disk_cache": bool(info["cg_from_disk_cache"]),
           "ms_per_eval": ms, "atom_steps_per_s": N / (ms * 1e-3), "status_flags": flags,
           "stage_ms_per_eval": {k: v / max(prof["calls"], 1) for k, v in prof.items() if k != "calls"}}
    if accuracy:
        # the FP64 engine on the same frame: absolute errors of the FP32 engine
        # (its CG kernel from the parallel build: the same results as the
        # one-program build, without the minute of single-threaded compile)
        pot64 = SUS2_SH(path, N, ["Cu", "Zr", "Al", "sus2_float=0", "sus2_sh_cg_whole=0", *opts])
        pe64, f64, w64 = z(N), z(3 * N), z(9 * N)
        pot64.compute(box, t, x, pe64, f64, w64)
        torch.cuda.synchronize()
        pot64.close()
        de = pe - pe64
        out["accuracy_fp32_vs_fp64"] = {
            "abs_dE_total_per_atom_eV": float(de.sum().abs()) / N, "site_dE_rms_eV": float((de ** 2).mean().sqrt()),
            "max_abs_site_dE_eV": float(de.abs().max()), "force_rms_eV_per_A": float(((f - f64) ** 2).mean().sqrt()),
            "virial_rms_eV": float(((w - w64) ** 2).mean().sqrt()),
            "site_energy_scale_eV": float(pe64.abs().max()), "force_rms_scale_eV_per_A": float((f64 ** 2).mean().sqrt())}
    return out


def cpu_baseline_leg(path, box, types, pos, engine_out):
    """The FP64 oracle (the reference's algorithm restated in C, OpenMP on all
    host cores) on the full final frame of the timed run: its throughput is
    the CPU baseline, and its energies, forces and virials are the checker of
    the FP32 engine's on the same frame (engine_out: pe[N], f[3,N], w[9,N])."""
    import numpy as np
    sys.path.insert(0, ORACLE)
    import sus2sh_oracle
    orc = sus2sh_oracle.Oracle(path)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    pe0, f0, w0 = orc.efs(box.cpu_h, box.pbc, types, pos, nthreads=threads)
    dt = time.perf_counter() - t0
    pe, f, w = engine_out
    de = pe - pe0
    accuracy = {"force_rms_fp32_vs_fp64_oracle_eV_per_A": float(np.sqrt(((f - f0) ** 2).mean())),
                "virial_rms_fp32_vs_fp64_oracle_eV": float(np.sqrt(((w - w0) ** 2).mean())),
                "abs_dE_total_per_atom_vs_oracle_eV": abs(float(de.sum())) / de.size,
                "site_dE_rms_vs_oracle_eV": float(np.sqrt((de ** 2).mean())),
                "max_abs_site_dE_vs_oracle_eV": float(np.abs(de).max())}
    baseline = {"value": types.size / dt, "unit": "atom-step/s", "cores": threads, "kind": "port",
                "sample": f"one FP64 oracle force evaluation of the full {types.size}-atom final frame of the "
                          f"timed run (same crystal and model), OpenMP {threads} threads"}
    return baseline, accuracy


MODEL_FIXTURE = os.path.join(REPO, "tests", "golden", "models", "l3k3.mtp")


def _reference_gpu_arm(args, path, box, types, pos):
    """The reference's own SUS2-SH engine (src/force/sus2_sh.cu, unmodified,
    nvcc sm_100a against minimal GPUMD stand-ins: oracle/_ref/ref_sus2sh) on
    the full workload frame, called as GPUMD's Force::compute calls it.  The
    reference rebuilds its neighbour list inside every call, so a call on a
    static frame costs what an MD step's force call costs; the integrator is
    not timed (it is GPUMD's)."""
    import numpy as np
    import ref_engine
    N = int(types.size)
    sym = ("Cu", "Zr")
    pe32, f32, w32, ms32, out32 = ref_engine.run(path, box.cpu_h, box.pbc, types, pos, sym, steps=args.steps,
                                                 warmup=args.warmup, timeout=1800)
    spread = {k: v for k, v in ref_engine.timing(out32).items() if k.startswith("ref_ms_")}
    k = max(1, min(args.steps, 10))
    _, _, _, _, out = ref_engine.run(path, box.cpu_h, box.pbc, types, pos,
                                     (*sym, "sus2_sh_profile=1", f"sus2_sh_profile_interval={k}"), steps=k,
                                     warmup=k, timeout=1800)
    stages = ref_engine.profile_stages(out)
    k64 = max(1, min(args.steps, 5))
    pe64, f64, _, ms64, _ = ref_engine.run(path, box.cpu_h, box.pbc, types, pos, (*sym, "sus2_float=0"), steps=k64,
                                           warmup=2, timeout=1800)
    value = N / (ms32 * 1e-3)
    sample = ("the reference's own CUDA engine (src/force/sus2_sh.cu, unmodified, nvcc sm_100a against minimal "
              "GPUMD stand-ins) on the full 1,024,000-atom frame on this GPU; the reference has no CPU path; "
              "one host thread drives it")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-step/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded FCC Cu-Zr, seeded random l3k3 model: tests/golden/models/l3k3.mtp)",
        "config": {"workload": "1.024M-atom l3k3 Cu-Zr (80x80x40 FCC, a=3.8 A, 64/36), SUS2_SH::compute per step",
                   "atoms": N, "inputs": "larger than L2 (positions 24.6 MB, moments 2 x 1 GB)"},
        "reference_build": "oracle/_ref/ref_sus2sh (src/force/sus2_sh.cu unmodified, sus2_float=1 default path)",
        "stage_ms_per_step": stages,
        "step_ms_spread": spread,
        "fp64": {"value": N / (ms64 * 1e-3), "ms_per_step": ms64, "steps": k64},
        "accuracy": {"force_rms_fp32_vs_fp64": float(np.sqrt(((f32 - f64) ** 2).mean())),
                     "max_site_energy_fp32_vs_fp64": float(np.abs(pe32 - pe64).max())},
        "cpu_baseline": {"value": value, "unit": "atom-step/s", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "atom-step/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def _reference_cpu_arm(args, path):
    """Without the reference build: the FP64 oracle port on this host's
    cores, one force evaluation of a 6,912-atom slice per step."""
    import sus2sh_oracle
    from sus2sh import structures
    box, types, pos = structures.fcc(12, 12, 12, A, (0.64, 0.36), 0.0, seed=7)
    orc = sus2sh_oracle.Oracle(path)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        orc.efs(box.cpu_h, box.pbc, types, pos, nthreads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.efs(box.cpu_h, box.pbc, types, pos, nthreads=threads)
    dt = time.perf_counter() - t0
    value = types.size * args.steps / dt
    sample = (f"one FP64 force evaluation per step of a {types.size}-atom 12^3-cell slice of the 1.024M-atom "
              f"FCC Cu-Zr crystal, same l3k3 model; reference-semantics C port, OpenMP {threads} threads")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "atom-step/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded FCC Cu-Zr, seeded random l3k3 model)",
            "config": {"workload": "1.024M-atom l3k3 Cu-Zr NVE (CPU arm: bounded per-step sample)",
                       "sample_atoms": int(types.size)},
            "cpu_baseline": {"value": value, "unit": "atom-step/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "atom-step/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_arm(args):
    """Rank 0 alone; loads no library of this repository (the model is the
    committed fixture, the structure plain numpy)."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, ORACLE)
    import ref_engine
    from sus2sh import structures
    import torch
    if ref_engine.available() and torch.cuda.is_available():
        box, types, pos = structures.fcc(*args.cells, A, (0.64, 0.36), 0.0, seed=1000)
        line = _reference_gpu_arm(args, MODEL_FIXTURE, box, types, pos)
    else:
        line = _reference_cpu_arm(args, MODEL_FIXTURE)
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.fp64_steps < 0:
        args.fp64_steps = args.steps
    if args.impl == "reference":
        reference_arm(args)
        return
    global CELLS_RUN
    CELLS_RUN = tuple(args.cells)
    import numpy as np
    import torch
    if args.large_only:
        with tempfile.TemporaryDirectory() as d:
            print(json.dumps({"large_model": large_model_run(torch, d, atoms=args.large_only)}), flush=True)
        return
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    from sus2sh import _lib
    lib = _lib.load()
    with tempfile.TemporaryDirectory() as d:
        path, box, types, pos, vel, masses = make_workload(d, rank)
        N = types.size
        clocks = ClockSampler(local)
        pot, md, ms, prof, launches, clk, frame = run_md(torch, path, box, types, pos, vel, masses, args.steps,
                                                  args.warmup, False, world, clocks)
        # FP64 engine on the same workload
        pot64 = md64 = None
        ms64 = None
        if args.fp64_steps > 0:
            pot64, md64, ms64, prof64, _, _, _ = run_md(torch, path, box, types, pos, vel, masses, args.fp64_steps,
                                                     min(args.warmup, 3), True, world)
        frms, de, de_total, final32 = force_error_vs_fp64(torch, path, box, types, frame)
        final_pos = frame.view(3, N).cpu().numpy()
        e2e_val, h2d, d2h = e2e_run(torch, pot, box, types, frame, args.e2e_steps)
        ms_max, ms64_max, inv_e2e = max_over_ranks(torch, [ms, ms64 or 0.0, 1.0 / max(e2e_val, 1e-30)], world,
                                                   "cuda")
        if rank == 0:
            value = whole_job_rate(N, world, args.steps, ms_max)
            info = pot.info()
            kmu = info["k_max"] * (info["l_max"] + 1)
            C = (info["l_max"] + 1) ** 2
            fb, ff, fp = flops_model(kmu, info["rb_size"], C, info["basics"], info["products"])
            edges = edges_within(box, pos, pot.rc)
            force_ms_launch = prof["force_ms"] / max(prof["calls"], 1)
            force_flops = edges * ff
            fp32_peak, fp64_peak = fma_peak()
            achieved = force_flops / (force_ms_launch * 1e-3) / 1e12
            step_flops = edges * (fb + ff) + N * fp
            line = {
                "metric": METRIC, "value": value, "unit": "atom-step/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded 80x80x40 FCC Cu-Zr 64/36, MB velocities 200 K; seeded random l3k3 model)",
                "config": {"workload": (f"{N / 1e6:.3f}M-atom" if N != 1024000 else "1.024M-atom")
                                       + " l3k3 Cu-Zr NVE MD, FP32 engine", "atoms_per_gpu": N,
                           "dt_fs": DT, "skin_A": SKIN, "rebuild_every": REBUILD, "rc_A": pot.rc,
                           "model": "SUS2-SH L3 K3 body4 rb8 (248 moments, 806 products)",
                           "l2": "inputs larger than L2 (positions+neighbour list+moments > 126 MB)",
                           "parallelism": f"replicas x{world}"},
                "fp64": {"value": whole_job_rate(N, world, args.fp64_steps, ms64_max) if ms64_max else None,
                         "ms_per_step": ms64_max / args.fp64_steps if ms64_max else None,
                         "steps": args.fp64_steps},
                "fp32_over_fp64": (value / whole_job_rate(N, world, args.fp64_steps, ms64_max)) if ms64_max else None,
                "accuracy": {"force_rms_fp32_vs_fp64_eV_per_A": frms, "max_abs_dE_per_atom_eV": de,
                             "abs_dE_total_per_atom_eV": de_total},
                "stage_ms_per_step": {k: v / max(prof["calls"], 1) for k, v in prof.items() if k != "calls"},
                "roofline": {"kernel": "k_force (adjoint force/virial; "
                                       + {0: "ahead-of-time build", 1: "NVRTC build of the shape",
                                          2: "NVRTC build specialised to the model"}.get(info["edge_jit"], "?")
                                       + f", {info['force_block']}-thread CTAs)", "bound": "fp32",
                             "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                             "frac": achieved / fp32_peak if fp32_peak > 0 else None,
                             "traffic": K_FORCE_DRAM_BYTES_PER_ATOM * N,
                             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_force on the "
                                               "524,288-atom case, scaled per atom",
                             "algorithmic_bytes": k_force_algorithmic_bytes(info["basics"], edges / N) * N,
                             "peak_source": "measured FP32 FMA-chain microbenchmark on this GPU (burst)",
                             "flops_per_edge": ff, "edges_per_launch": edges,
                             "launch_ms": force_ms_launch,
                             "step_tflops": step_flops * args.steps / (ms_max * 1e-3) / 1e12 / world,
                             "fp64_peak_tflops": fp64_peak},
                "e2e": {"value": 1.0 / inv_e2e * world, "unit": "atom-step/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h,
                        "path": "sus2sh_compute_host: pinned host positions -> device -> energies/forces/virial "
                                "-> pinned host, every step"},
                "gpu_launches": launches,
                "clocks": clk,
            }
            if world == 1 and not args.no_extra:
                line["batch_cells"] = batch_cells_run(torch, path)
                line["large_model"] = lm = large_model_run(torch, d)
                # the component-split CG kernel against the FP32 peak: the
                # counting rule's 9 flop per product (3 forward, 6 reverse)
                prod_ms = lm["stage_ms_per_eval"].get("product_ms", 0.0)
                if prod_ms > 0 and fp32_peak > 0:
                    tf = lm["atoms"] * 9 * 33389 / (prod_ms * 1e-3) / 1e12
                    lm["product_roofline"] = {"kernel": "component-split CG kernel", "bound": "fp32",
                                              "achieved": tf, "peak": fp32_peak, "unit": "TFLOP/s",
                                              "frac": tf / fp32_peak,
                                              "flop_rule": "9 per product per atom (33,389 products)"}
            if world == 1 and not args.no_cpu_baseline:
                line["cpu_baseline"], acc_oracle = cpu_baseline_leg(path, box, types, final_pos, final32)
                line["accuracy"].update(acc_oracle)
            print(json.dumps(line), flush=True)
        pot.close()
        if pot64:
            pot64.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
