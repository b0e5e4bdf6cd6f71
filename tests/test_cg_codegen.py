"""The model-specialised CG kernels are generated and NVRTC-compiled for sm_100a
at model load (no GPU needed to compile).  Small graphs get one straight-line
function; large graphs the component-split kernel.  The generated source of
either is also compiled with the host C++ compiler and run on random basic
moments, and its site energies and basic adjoints are compared with the FP64
oracle's flat CG evaluation (oracle_cg_energy, the algorithm of
src/force/sus2_sh.cu:4799-4846)."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import sus2sh_oracle as O
from sus2sh import _lib, models

FIELDS = ("regs", "spill", "terms", "ms", "cubin", "split", "functions", "components", "block", "smem")


def _info(path, use_float, split=-1, text_size=8192):
    lib = _lib.load()
    info = (ctypes.c_int * len(FIELDS))()
    txt = ctypes.create_string_buffer(text_size)
    rc = lib.sus2sh_cg_kernel_info(path.encode(), use_float, split, info, txt, text_size)
    return rc, dict(zip(FIELDS, list(info))), txt.value.decode()


def test_l3k3_cg_kernel_compiles_without_spills(l3k3_path):
    rc, info, log = _info(l3k3_path, 1)
    assert rc == 0, log
    assert info["split"] == 0 and info["functions"] == 1
    assert 0 < info["regs"] <= 255 and info["spill"] == 0, log
    # 806 products: 606 forward terms + 200 fused terminal terms (x2) + 606 back terms (x2)
    assert info["terms"] == 606 + 2 * 200 + 2 * 606
    assert info["cubin"] > 0


def test_fused_batch_kernel_compiles_without_spills(l3k3_path, l4k4_path):
    """The fused persistent batch kernel of the l3k3 model (moments, the
    straight-line CG contraction and the force loop in one kernel) builds
    without a GPU: the 3-CTA-per-SM variant stays within 170 registers and
    neither variant spills.  A graph that takes the component-split CG kernel
    has no fused kernel (its batches always run the stage kernels)."""
    lib = _lib.load()
    info = (ctypes.c_int * 4)()
    log = ctypes.create_string_buffer(1 << 16)
    rc = lib.sus2sh_batch_kernel_info(l3k3_path.encode(), info, log, len(log))
    assert rc == 0, lib.sus2sh_last_error().decode()
    assert 0 < info[0] <= 170 and 0 < info[1] <= 255 and info[3] > 0
    text = log.value.decode()
    assert len(re.findall(r"Compiling entry function '\w*k_batch_fused", text)) == 2
    assert "bytes spill stores" in text and not re.search(r"[1-9]\d* bytes spill stores", text), text
    rc = lib.sus2sh_batch_kernel_info(l4k4_path.encode(), info, None, 0)
    assert rc == -1 and "component-split" in lib.sus2sh_last_error().decode()


def test_large_graph_gets_the_split_kernel(l4k4_path):
    # l4k4 body 5: 33,389 products in 116 (rank L, component M) components
    # (split=3: the parallel relocatable build, seconds instead of the
    # one-program build's minute on the host)
    rc, info, log = _info(l4k4_path, 1, split=3)
    assert rc == 0, _lib.load().sus2sh_last_error().decode()
    assert info["split"] == 1 and info["components"] == 116
    assert info["block"] == 128 and info["smem"] == 2 * 100 * 128 * 4
    assert info["spill"] == 0, log


_CACHE_PROBE = r"""
import ctypes, sys
sys.path.insert(0, sys.argv[1])
from sus2sh import _lib
lib = _lib.load()
info = (ctypes.c_int * 10)()
rc = lib.sus2sh_cg_kernel_info(sys.argv[2].encode(), 1, int(sys.argv[3]), info, None, 0)
print(rc, info[3], info[4])
"""


def _probe(path, split, cache_dir):
    env = dict(os.environ, SUS2SH_CACHE_DIR=cache_dir)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpumd-sus2-sh_b200")
    out = subprocess.run([sys.executable, "-c", _CACHE_PROBE, pkg, path, str(split)], env=env, check=True,
                         capture_output=True, text=True).stdout.split()
    return int(out[0]), int(out[1]), int(out[2])


@pytest.mark.parametrize("split", [-1, 1], ids=["straight_line", "component_split"])
def test_one_program_builds_go_through_the_disk_cache(l3k3_path, tmp_path, split):
    # each process starts with an empty in-process cache: the first compiles
    # and writes the cubin, the second reads it back, a damaged file is
    # ignored and rewritten
    cache = str(tmp_path / "cache")
    rc, ms_first, size = _probe(l3k3_path, split, cache)
    assert rc == 0 and size > 0
    files = [f for f in os.listdir(cache) if f.startswith("cg_") and f.endswith(".cubin")]
    assert len(files) == 1
    fpath = os.path.join(cache, files[0])
    with open(fpath, "rb") as f:
        blob = f.read()
    assert blob[:8] == b"SUS2CGB1" and len(blob) > size
    rc, ms_cached, size2 = _probe(l3k3_path, split, cache)
    assert rc == 0 and size2 == size and ms_cached < max(50, ms_first // 4), (ms_first, ms_cached)
    with open(fpath, "wb") as f:
        f.write(blob[: len(blob) // 2])  # truncated
    rc, _, size3 = _probe(l3k3_path, split, cache)
    assert rc == 0 and size3 == size
    with open(fpath, "rb") as f:
        again = f.read()  # rewritten whole (NVRTC output is not byte-stable: compare the header and length)
    assert len(again) == len(blob) and again[:40] == blob[:40] and again[48:64] == blob[48:64]
    assert not [f for f in os.listdir(cache) if ".tmp" in f]
    rc, _, size4 = _probe(l3k3_path, split, "off")  # disabled
    assert rc == 0 and size4 == size


def test_large_graph_without_split_runs_the_interpreter(l4k4_path):
    rc, _, _ = _info(l4k4_path, 1, split=0)
    assert rc == -1
    assert "interpreter" in _lib.load().sus2sh_last_error().decode()


# ---------------------------------------------------------------------------
# host emulation of the generated CUDA source
# ---------------------------------------------------------------------------
_PRELUDE = r"""
#include <cmath>
#include <cstddef>
#include <cstring>
#define __device__
#define __noinline__ __attribute__((noinline))
#define __global__
#define __launch_bounds__(...)
#define __shared__
#define __align__(n) __attribute__((aligned(n)))
#define __syncthreads()
struct EmuDim { unsigned x; };
static EmuDim threadIdx, blockIdx, blockDim;
template <class T> static inline T __ldg(const T* p) { return *p; }
static inline unsigned long long sus2_pol() { return 0; }
template <class T> static inline T sus2_ld(const T* p, unsigned long long) { return *p; }
template <class T> static inline void sus2_st(T* p, T v, unsigned long long) { *p = v; }
static inline long long __double_as_longlong(double d) { long long v; std::memcpy(&v, &d, 8); return v; }
using std::fma;
using std::fmaf;
unsigned char smem_raw[232448] __attribute__((aligned(16)));
"""

_DRIVER = r"""
extern "C" void run(int N, int block, const float* B, float* G, const int* type, const double* shift,
                    const double* species, double* pe) {
  D4* p4 = new D4[N];
  for (int i = 0; i < N; ++i) {
    long long t = type[i];
    double w;
    std::memcpy(&w, &t, 8);
    p4[i] = D4{0, 0, 0, w};
  }
  blockDim.x = block;
  for (int i = 0; i < N; ++i) {  // one lane at a time: every lane owns its shared-memory column
    threadIdx.x = i % block;
    blockIdx.x = i / block;
    KERNEL(N, p4, B, G, shift, species, pe, 1);
  }
  delete[] p4;
}
"""


def _emulate(path, split, tmp_path, N=45, seed=3):
    rc, info, src = _info(path, -1, split=split, text_size=1 << 26)   # use_float < 0: FP32 source text
    assert rc == 0, _lib.load().sus2sh_last_error().decode()
    name = re.search(r"(sus2sh_cg\w+)\(int N", src).group(1)
    block = info["block"]
    canon = dict((int(b), int(c)) for b, c in re.findall(r"(?:sv\[|v)(\d+)(?: \* \d+\])? = sus2_ld\(B \+ (\d+) \* n", src))
    cpp = tmp_path / "k.cpp"
    cpp.write_text(_PRELUDE + src.replace('extern "C" __global__', "__global__") + _DRIVER.replace("KERNEL", name))
    so = tmp_path / "k.so"
    subprocess.check_call(["g++", "-O1", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(so), str(cpp)])
    lib = ctypes.CDLL(str(so))
    orc = O.Oracle(path)
    m = orc.model
    rng = np.random.default_rng(seed)
    nb = m.alpha_basic_count
    Bm = rng.normal(0.0, 1.0, (nb, N))
    types = rng.integers(0, m.species_count, N).astype(np.int32)
    pe0, G0 = orc.cg_energy(types, Bm)
    ncanon = max(canon.values()) + 1
    Bc = np.zeros((ncanon, N), np.float32)
    for b, c in canon.items():
        Bc[c] = Bm[b]
    Gc = np.zeros((ncanon, N), np.float32)
    pe = np.zeros(N)
    shift = np.ascontiguousarray(m.shift_coeffs, dtype=np.float64)
    species = np.ascontiguousarray(m.species_coeffs, dtype=np.float64)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib.run(N, block, P(Bc), P(Gc), P(types), P(shift), P(species), P(pe))
    G = np.array([Gc[canon[b]] for b in range(nb)], dtype=np.float64)
    scale = max(1.0, np.abs(pe0 - shift[types]).max())
    return np.abs(pe - pe0).max() / scale, np.abs(G - G0).max() / np.abs(G0).max(), info


@pytest.mark.parametrize("split", [0, 1])
def test_generated_kernels_match_oracle_on_host(l3k3_path, tmp_path, split):
    de, dg, info = _emulate(l3k3_path, split, tmp_path)
    assert info["split"] == split
    assert de < 1e-6 and dg < 1e-5, (de, dg)


@pytest.fixture(scope="module")
def body5_path(tmp_path_factory):
    # l3k3 body 5: 5,475 products, above the single-function limit
    p = str(tmp_path_factory.mktemp("models") / "l3k3b5.mtp")
    return models.write_model(p, species=2, l_max=3, k_max=3, body_order=5, rb_size=8, seed=11)


@pytest.fixture(scope="module")
def body6_path(tmp_path_factory):
    # l2k2 body 6: three layers, shared intermediates feed non-terminal rows
    p = str(tmp_path_factory.mktemp("models") / "l2k2b6.mtp")
    return models.write_model(p, species=2, l_max=2, k_max=2, body_order=6, rb_size=8, seed=12)


def test_split_kernel_body5_matches_oracle_on_host(body5_path, tmp_path):
    de, dg, info = _emulate(body5_path, -1, tmp_path)
    assert info["split"] == 1 and info["components"] == 64
    assert de < 1e-6 and dg < 1e-5, (de, dg)


def test_split_kernel_body6_shared_intermediates_on_host(body6_path, tmp_path):
    de, dg, info = _emulate(body6_path, 1, tmp_path)
    assert info["split"] == 1
    assert info["smem"] > 2 * 18 * info["block"] * 4   # 18 basics + shared intermediates
    assert de < 1e-6 and dg < 1e-5, (de, dg)


# ---------------------------------------------------------------------------
# forward-over-reverse product kernel of the parameter gradients
# ---------------------------------------------------------------------------
_PG_DRIVER = r"""
extern "C" void run_pg(int N, int block, const float* B, const float* Bd, const int* type, const double* species,
                       const double* ew, float* Ga, float* Gb, float* contrib) {
  D4* p4 = new D4[N];
  for (int i = 0; i < N; ++i) {
    long long t = type[i];
    double w;
    std::memcpy(&w, &t, 8);
    p4[i] = D4{0, 0, 0, w};
  }
  blockDim.x = block;
  for (int i = 0; i < N; ++i) {
    threadIdx.x = i % block;
    blockIdx.x = i / block;
    KERNEL(N, p4, B, Bd, species, ew, Ga, Gb, contrib);
  }
  delete[] p4;
}
"""


def _flat_dual(m, types, Bm, Bdm, ew):
    """Flat products in file order with dual numbers (the interpreter's
    algorithm): returns alpha, beta per basic and contrib per scalar."""
    N = Bm.shape[1]
    M = m.alpha_moments_count
    nb = m.alpha_basic_count
    Mv = np.zeros((M, N)); Md = np.zeros((M, N))
    Mv[:nb] = Bm; Md[:nb] = Bdm
    for (l, r, t, c) in m.products:
        Md[t] += c * (Md[l] * Mv[r] + Mv[l] * Md[r])
        Mv[t] += c * Mv[l] * Mv[r]
    ct = np.asarray(m.species_coeffs)[types]
    gv = np.zeros((M, N)); gd = np.zeros((M, N))
    contrib = np.zeros((m.alpha_scalar_moments, N))
    for s, (mm, w) in enumerate(zip(m.alpha_moment_mapping, m.moment_coeffs)):
        gv[mm] += ct * w
        contrib[s] = ct * (ew * Mv[mm] - Md[mm])
    for (l, r, t, c) in reversed(m.products):
        gt, gdt = c * gv[t], c * gd[t]
        gd[l] += gdt * Mv[r] + gt * Md[r]
        gd[r] += gdt * Mv[l] + gt * Md[l]
        gv[l] += gt * Mv[r]
        gv[r] += gt * Mv[l]
    return ew * gv[:nb] - gd[:nb], gv[:nb], contrib


def test_param_grad_product_kernel_matches_flat_duals_on_host(l3k3_path, tmp_path):
    rc, info, src = _info(l3k3_path, -1, split=2, text_size=1 << 26)
    assert rc == 0, _lib.load().sus2sh_last_error().decode()
    name = re.search(r"(sus2sh_pg_\w+)\(int N", src).group(1)
    canon = dict((int(b), int(c)) for b, c in re.findall(r"v(\d+) = __ldg\(B \+ (\d+) \* n \+ i\)", src))
    cpp = tmp_path / "pg.cpp"
    cpp.write_text(_PRELUDE + src.replace('extern "C" __global__', "__global__") + _PG_DRIVER.replace("KERNEL", name))
    so = tmp_path / "pg.so"
    subprocess.check_call(["g++", "-O1", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(so), str(cpp)])
    lib = ctypes.CDLL(str(so))
    m = O.Oracle(l3k3_path).model
    N = 37
    rng = np.random.default_rng(9)
    nb = m.alpha_basic_count
    Bm = rng.normal(0.0, 1.0, (nb, N))
    Bdm = rng.normal(0.0, 0.3, (nb, N))
    types = rng.integers(0, m.species_count, N).astype(np.int32)
    ew = rng.normal(0.0, 1.0, N)
    al0, be0, co0 = _flat_dual(m, types, Bm, Bdm, ew)
    ncanon = max(canon.values()) + 1
    Bc = np.zeros((ncanon, N), np.float32)
    Bdc = np.zeros((ncanon, N), np.float32)
    for b, c in canon.items():
        Bc[c] = Bm[b]
        Bdc[c] = Bdm[b]
    Ga = np.zeros((ncanon, N), np.float32)
    Gb = np.zeros((ncanon, N), np.float32)
    co = np.zeros((m.alpha_scalar_moments, N), np.float32)
    species = np.ascontiguousarray(m.species_coeffs, dtype=np.float64)
    ewc = np.ascontiguousarray(ew)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib.run_pg(N, 128, P(Bc), P(Bdc), P(types), P(species), P(ewc), P(Ga), P(Gb), P(co))
    al = np.array([Ga[canon[b]] for b in range(nb)], dtype=np.float64)
    be = np.array([Gb[canon[b]] for b in range(nb)], dtype=np.float64)
    rel = lambda x, y: np.abs(x - y).max() / max(np.abs(y).max(), 1e-30)
    assert rel(al, al0) < 2e-5 and rel(be, be0) < 2e-5, (rel(al, al0), rel(be, be0))
    assert rel(co.astype(np.float64), co0) < 2e-5, rel(co.astype(np.float64), co0)
