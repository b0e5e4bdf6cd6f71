"""Oracle (test infrastructure only): Python front end of the FP64 C oracle
``sus2sh_oracle.c`` plus a pure-Python evaluator for tiny cases.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module.  The model is read by ``sus2sh_graph.load_mtp``
(the restated reference reader), never by the product library, so the oracle
and the product share no code.

Radial tables are FP64 (the reference rounds them to FP32 even in its
``sus2_float=0`` path, src/force/sus2_sh.cu:2484-2517); pass
``reference_rounding=True`` to reproduce that rounding for an A/B.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

from sus2sh_graph import MtpModel, load_mtp  # noqa: F401  (re-exported)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build_oracle(force: bool = False) -> str:
    """Compiles the C oracle (gcc, OpenMP) next to this file."""
    src = os.path.join(_HERE, "sus2sh_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", _LIB_PATH, src, "-lm"])
    return _LIB_PATH


class _COracleModel(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ("S", "L", "K", "rb", "kmu", "M", "nbasic", "nscalar", "nprod", "kind")] + [
        ("rc", ctypes.c_double),
        ("radial", ctypes.c_void_p), ("scal", ctypes.c_void_p), ("rshift", ctypes.c_void_p),
        ("pscale", ctypes.c_void_p), ("basic_mu", ctypes.c_void_p), ("basic_y", ctypes.c_void_p),
        ("prod_l", ctypes.c_void_p), ("prod_r", ctypes.c_void_p), ("prod_t", ctypes.c_void_p),
        ("prod_c", ctypes.c_void_p), ("map", ctypes.c_void_p), ("w", ctypes.c_void_p),
        ("shift_e", ctypes.c_void_p), ("species", ctypes.c_void_p)]


@dataclass
class OracleArrays:
    """Flat FP64/int32 arrays of a model, as the C oracle consumes them."""
    model: MtpModel
    radial: np.ndarray
    scal: np.ndarray
    rshift: np.ndarray
    pscale: np.ndarray
    basic_mu: np.ndarray
    basic_y: np.ndarray
    prod_l: np.ndarray
    prod_r: np.ndarray
    prod_t: np.ndarray
    prod_c: np.ndarray
    map: np.ndarray
    w: np.ndarray
    shift_e: np.ndarray
    species: np.ndarray

    @classmethod
    def from_model(cls, m: MtpModel, reference_rounding: bool = False) -> "OracleArrays":
        S, kmu = m.species_count, m.radial_funcs_count
        f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if reference_rounding else (lambda a: a)
        radial = f32(np.asarray(m.radial_coeffs, dtype=np.float64))
        scal = np.zeros((S * S, kmu))
        rsh = np.zeros((S * S, kmu))
        ps = np.zeros(S * S)
        sc = np.asarray(m.scal_coeffs, dtype=np.float64)
        for zi in range(S):
            for zj in range(S):
                p = zi * S + zj
                for mu in range(kmu):
                    off = 2 * mu * S * S + S * zi + zj
                    scal[p, mu] = sc[off]
                    rsh[p, mu] = sc[off + S * S]
                ps[p] = m.scaling * m.radial_type_coeffs[zi] * m.radial_type_coeffs[zj]
        basic_mu = np.array([b[0] for b in m.alpha_basic], dtype=np.int32)
        basic_y = np.array([b[1] * b[1] + b[1] + b[2] for b in m.alpha_basic], dtype=np.int32)
        P = np.array(m.products, dtype=np.float64).reshape(-1, 4)
        return cls(m, radial, f32(scal.ravel()), f32(rsh.ravel()), f32(ps), basic_mu, basic_y,
                   P[:, 0].astype(np.int32), P[:, 1].astype(np.int32), P[:, 2].astype(np.int32),
                   np.ascontiguousarray(P[:, 3]),
                   np.asarray(m.alpha_moment_mapping, dtype=np.int32),
                   np.asarray(m.moment_coeffs, dtype=np.float64),
                   np.asarray(m.shift_coeffs, dtype=np.float64),
                   np.asarray(m.species_coeffs, dtype=np.float64))

    def c_struct(self) -> _COracleModel:
        m = self.model
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        return _COracleModel(m.species_count, m.sh_l_max, m.sh_k_max, m.rb_size, m.radial_funcs_count,
                             m.alpha_moments_count, m.alpha_basic_count, len(self.map), len(self.prod_c),
                             2 if m.laguerre else (1 if m.rational else 0), m.max_dist,
                             ptr(self.radial), ptr(self.scal), ptr(self.rshift), ptr(self.pscale),
                             ptr(self.basic_mu), ptr(self.basic_y), ptr(self.prod_l), ptr(self.prod_r),
                             ptr(self.prod_t), ptr(self.prod_c), ptr(self.map), ptr(self.w),
                             ptr(self.shift_e), ptr(self.species))


_ELEMENTS = ("H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se "
             "Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb "
             "Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu").split()

_ZBL_TABLE_ERRORS = {
    1: "ZBL requires one atomic number per model species.",
    2: "ZBL inner cutoff should be non-negative.",
    3: "ZBL outer cutoff should be positive.",
    4: "ZBL typewise cutoff factor should be at least 0.5.",
    5: "ZBL cutoffs should satisfy 0 <= inner < outer.",
    6: "ZBL atomic numbers should be in [1, 94].",
    7: "ZBL pair cutoffs should satisfy inner < outer.",
}


def atomic_number(symbol: str) -> int:
    """sus2_zbl_atomic_number_from_symbol (sus2_zbl_common.cuh:54-71); 0 if unknown."""
    return _ELEMENTS.index(symbol) + 1 if symbol in _ELEMENTS else 0


def zbl_tables(z, inner: float, outer: float, typewise: bool, factor: float):
    """Pair inner/outer cutoffs [S*S] (sus2_zbl_fill_pair_cutoff_tables,
    sus2_zbl_common.cuh:89-169) through the C restatement; ValueError with the
    reference's message on a failed check."""
    lib = ctypes.CDLL(build_oracle())
    S = len(z)
    za = np.ascontiguousarray(np.asarray(z, dtype=np.int32))
    pin = np.zeros(max(S * S, 1))
    pout = np.zeros(max(S * S, 1))
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib.oracle_zbl_tables(S, ptr(za), ctypes.c_double(inner), ctypes.c_double(outer), int(typewise),
                               ctypes.c_double(factor), ptr(pin), ptr(pout))
    if rc != 0:
        raise ValueError(_ZBL_TABLE_ERRORS[rc])
    return pin[:S * S], pout[:S * S]


def zbl_pair(zi: int, zj: int, r: float, inner: float, outer: float):
    """Energy and dE/dr of one ZBL pair (C restatement)."""
    lib = ctypes.CDLL(build_oracle())
    e, de = ctypes.c_double(), ctypes.c_double()
    lib.oracle_zbl_pair(zi, zj, ctypes.c_double(r), ctypes.c_double(inner), ctypes.c_double(outer),
                        ctypes.byref(e), ctypes.byref(de))
    return e.value, de.value


class _COracleGate(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("nbody", ctypes.c_int), ("nq", ctypes.c_int),
                ("amplitude", ctypes.c_double),
                ("radial", ctypes.c_void_p), ("additive", ctypes.c_void_p), ("q_moment", ctypes.c_void_p),
                ("q_body", ctypes.c_void_p), ("weights", ctypes.c_void_p), ("body_mix", ctypes.c_void_p)]


class Oracle:
    """FP64 energy/force/virial of one model (C oracle, OpenMP).  ZBL models
    take their atomic numbers from ``zbl_atomic_numbers`` or, as the
    reference's constructor does (sus2_sh.cu:7824-7860), from ``symbols``."""

    def __init__(self, model_or_path, reference_rounding: bool = False, symbols=None):
        m = load_mtp(model_or_path) if isinstance(model_or_path, str) else model_or_path
        self.model = m
        self.arrays = OracleArrays.from_model(m, reference_rounding)
        self._c = self.arrays.c_struct()
        self.lib = ctypes.CDLL(build_oracle())
        self.lib.oracle_efs.restype = ctypes.c_int
        self.lib.oracle_basics.restype = ctypes.c_int
        self.lib.oracle_neighbor_counts.restype = ctypes.c_int
        self.gate = None
        if m.gate is not None:
            g = m.gate
            f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if reference_rounding else (lambda a: a)
            arrs = dict(radial=f32(np.asarray(g["radial"], dtype=np.float64)),
                        additive=np.asarray(g["additive"], dtype=np.float64),
                        q_moment=np.asarray(g["moment_of"], dtype=np.int32),
                        q_body=np.asarray(g["body_of"], dtype=np.int32),
                        weights=np.asarray(g["weights"], dtype=np.float64),
                        body_mix=np.asarray(g["body_mix"] or [0.0], dtype=np.float64))
            ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
            self._gate_arrays = arrs
            self.gate = _COracleGate(g["mode"], g["nbody"], len(g["moment_of"]), g["amplitude"],
                                     *(ptr(arrs[k]) for k in ("radial", "additive", "q_moment", "q_body",
                                                              "weights", "body_mix")))
        self.zbl = None
        if m.zbl_enabled:
            z = m.zbl_atomic_numbers
            if not z:
                if symbols is None or len(symbols) < m.species_count:
                    raise ValueError("SUS2_SH ZBL model requires zbl_atomic_numbers metadata or element "
                                     "symbols after the model file.")
                z = [atomic_number(sym) for sym in symbols[:m.species_count]]
                if min(z) <= 0:
                    raise ValueError("SUS2_SH ZBL cannot map element symbol to an atomic number")
            if len(z) != m.species_count:
                raise ValueError("SUS2_SH ZBL metadata should provide one atomic number per species.")
            pin, pout = zbl_tables(z, m.zbl_inner, m.zbl_outer, m.zbl_typewise,
                                   m.zbl_typewise_factor if m.zbl_typewise else 0.0)
            self.zbl = (np.asarray(z, dtype=np.int32), pin, pout)

    def efs(self, h, pbc, types, pos, nthreads: int = 0):
        """Per-atom energy (N), forces (3, N) and virial (9, N); ``pos`` is (3, N)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        N = pos.shape[1]
        types = np.ascontiguousarray(types, dtype=np.int32)
        h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).ravel())
        pbc = np.ascontiguousarray(np.asarray(pbc, dtype=np.int32))
        pe = np.zeros(N)
        f = np.zeros((3, N))
        vir = np.zeros((9, N))
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        if self.gate is not None:
            rc = self.lib.oracle_efs_gate(ctypes.byref(self._c), ctypes.byref(self.gate), N, ptr(h), ptr(pbc),
                                          ptr(types), ptr(pos), ptr(pe), ptr(f), ptr(vir), nthreads)
        else:
            rc = self.lib.oracle_efs(ctypes.byref(self._c), N, ptr(h), ptr(pbc), ptr(types), ptr(pos),
                                     ptr(pe), ptr(f), ptr(vir), nthreads)
        if rc != 0:
            raise RuntimeError("oracle_efs failed")
        if self.zbl is not None:
            z, pin, pout = self.zbl
            if self.lib.oracle_zbl_efs(self.model.species_count, ptr(z), ptr(pin), ptr(pout), N, ptr(h),
                                       ptr(pbc), ptr(types), ptr(pos), ptr(pe), ptr(f), ptr(vir), nthreads) != 0:
                raise RuntimeError("oracle_zbl_efs failed")
        return pe, f, vir

    def efs_centers(self, h, pbc, types, pos, center, nthreads: int = 0):
        """As efs, but only atoms with center != 0 are centres (site energies,
        the forces of those energies on every atom, their virials); the other
        atoms get zero energy and virial.  Plain models (no gate, no ZBL)."""
        if self.gate is not None or self.zbl is not None:
            raise ValueError("efs_centers: plain models only")
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        N = pos.shape[1]
        types = np.ascontiguousarray(types, dtype=np.int32)
        h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).ravel())
        pbc = np.ascontiguousarray(np.asarray(pbc, dtype=np.int32))
        mask = np.ascontiguousarray(np.asarray(center) != 0, dtype=np.uint8)
        pe, f, vir = np.zeros(N), np.zeros((3, N)), np.zeros((9, N))
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        if self.lib.oracle_efs_centers(ctypes.byref(self._c), N, ptr(h), ptr(pbc), ptr(types), ptr(pos), ptr(mask),
                                       ptr(pe), ptr(f), ptr(vir), nthreads) != 0:
            raise RuntimeError("oracle_efs_centers failed")
        return pe, f, vir

    def basics(self, h, pbc, types, pos, nthreads: int = 0):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        N = pos.shape[1]
        types = np.ascontiguousarray(types, dtype=np.int32)
        h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).ravel())
        pbc = np.ascontiguousarray(np.asarray(pbc, dtype=np.int32))
        B = np.zeros((self.model.alpha_basic_count, N))
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        if self.lib.oracle_basics(ctypes.byref(self._c), N, ptr(h), ptr(pbc), ptr(types), ptr(pos),
                                  ptr(B), nthreads) != 0:
            raise RuntimeError("oracle_basics failed")
        return B


    def cg_energy(self, types, B):
        """Site energies and dE_i/dB_b(i) from basic moments B (model order, (Bb, N))."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        N = B.shape[1]
        types = np.ascontiguousarray(types, dtype=np.int32)
        pe = np.zeros(N)
        G = np.zeros_like(B)
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        if self.lib.oracle_cg_energy(ctypes.byref(self._c), N, ptr(types), ptr(B), ptr(pe), ptr(G)) != 0:
            raise RuntimeError("oracle_cg_energy failed")
        return pe, G


def neighbor_counts(h, pbc, pos, rc):
    lib = ctypes.CDLL(build_oracle())
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    N = pos.shape[1]
    h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).ravel())
    pbc = np.ascontiguousarray(np.asarray(pbc, dtype=np.int32))
    out = np.zeros(N, dtype=np.int32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    if lib.oracle_neighbor_counts(N, ptr(h), ptr(pbc), ptr(pos), ctypes.c_double(rc), ptr(out)) != 0:
        raise RuntimeError("oracle_neighbor_counts failed")
    return out


# ---------------------------------------------------------------------------
# Pure-Python evaluator (tiny cases only): brute-force images, flat products.
# Independent of the C oracle; used to cross-check it.
# ---------------------------------------------------------------------------

_YNORM = [0.5 / math.sqrt(math.pi)] + [0.5 * math.sqrt(3 / math.pi)] * 3


def real_sh_from_complex(l: int, m: int, d) -> float:
    """Real Y_lm built from the complex harmonic with the Condon-Shortley phase
    (scipy-free): Y_l0 = Y_l^0, Y_lm = sqrt2 (-1)^m Re Y_l^m (m>0),
    Y_l,-|m| = sqrt2 (-1)^m Im Y_l^|m|.  Pins the basis convention."""
    x, y, z = d
    r = math.sqrt(x * x + y * y + z * z)
    theta = math.acos(max(-1.0, min(1.0, z / r)))
    phi = math.atan2(y, x)
    am = abs(m)
    # associated Legendre with Condon-Shortley phase
    ct = math.cos(theta)
    st = math.sin(theta)
    pmm = 1.0
    for i in range(1, am + 1):
        pmm *= -(2 * i - 1) * st
    if l == am:
        plm = pmm
    else:
        pm1 = ct * (2 * am + 1) * pmm
        if l == am + 1:
            plm = pm1
        else:
            p0, p1 = pmm, pm1
            for ll in range(am + 2, l + 1):
                p0, p1 = p1, ((2 * ll - 1) * ct * p1 - (ll + am - 1) * p0) / (ll - am)
            plm = p1
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    if m == 0:
        return norm * plm
    sign = -1.0 if am % 2 else 1.0
    if m > 0:
        return math.sqrt(2) * sign * norm * plm * math.cos(am * phi)
    return math.sqrt(2) * sign * norm * plm * math.sin(am * phi)


def python_efs(m: MtpModel, h, pbc, types, pos, reach=2):
    """Energy, forces, virial by the flat reference algorithm, pure Python,
    with harmonics from ``real_sh_from_complex`` and central-difference
    derivatives of R and Y (step 1e-6) -- slow, independent, tiny N only."""
    N = pos.shape[1]
    S, kmu, rb, rc = m.species_count, m.radial_funcs_count, m.rb_size, m.max_dist
    hm = np.asarray(h, dtype=float).reshape(3, 3)

    def radial(pair, r):
        zi, zj = divmod(pair, S)
        out = []
        for mu in range(kmu):
            off = 2 * mu * S * S + S * zi + zj
            sc, sh = m.scal_coeffs[off], m.scal_coeffs[off + S * S]
            env = 1.0
            if m.laguerre:
                u = sc * math.log1p(r / max(sh, 1e-8))
                env = math.exp(-0.5 * u)
                t = [1.0, 1.0 - u]
                for n in range(1, rb - 1):
                    t.append(((2 * n + 1 - u) * t[n] - n * t[n - 1]) / (n + 1))
            else:
                z = 0.5 * sc * (r - sh)
                xi = z / math.sqrt(1 + z * z) if m.rational else math.tanh(z)
                t = [1.0, xi]
                for n in range(2, rb):
                    t.append(2 * xi * t[-1] - t[-2])
            s = sum(m.radial_coeffs[mu * rb + n] * t[n] for n in range(rb))
            out.append(m.scaling * m.radial_type_coeffs[zi] * m.radial_type_coeffs[zj] * (r - rc) ** 2 * env * s)
        return out

    def edge_basics(pair, d):
        r = math.sqrt(sum(c * c for c in d))
        R = radial(pair, r)
        return [R[mu] * real_sh_from_complex(l, mm, d) for (mu, l, mm) in m.alpha_basic]

    edges = [[] for _ in range(N)]
    rng = range(-reach, reach + 1)
    for i in range(N):
        for j in range(N):
            for tx in (rng if pbc[0] else [0]):
                for ty in (rng if pbc[1] else [0]):
                    for tz in (rng if pbc[2] else [0]):
                        if i == j and tx == ty == tz == 0:
                            continue
                        d = pos[:, j] - pos[:, i] + hm @ np.array([tx, ty, tz], dtype=float)
                        if float(d @ d) < rc * rc:
                            edges[i].append((j, d.copy()))
    pe = np.zeros(N)
    f = np.zeros((3, N))
    vir = np.zeros((9, N))
    for i in range(N):
        ti = int(types[i])
        Mv = [0.0] * m.alpha_moments_count
        for j, d in edges[i]:
            for b, v in enumerate(edge_basics(ti * S + int(types[j]), d)):
                Mv[b] += v
        for (l, r_, t, c) in m.products:
            Mv[t] += c * Mv[l] * Mv[r_]
        ct = m.species_coeffs[ti]
        pe[i] = m.shift_coeffs[ti] + ct + ct * sum(w * Mv[s] for s, w in zip(m.alpha_moment_mapping, m.moment_coeffs))
        g = [0.0] * m.alpha_moments_count
        for s, w in zip(m.alpha_moment_mapping, m.moment_coeffs):
            g[s] += ct * w
        for (l, r_, t, c) in reversed(m.products):
            gt = g[t] * c
            g[l] += gt * Mv[r_]
            g[r_] += gt * Mv[l]
        for j, d in edges[i]:
            dE = np.zeros(3)
            eps = 1e-6
            for a in range(3):
                dp = d.copy(); dp[a] += eps
                dm = d.copy(); dm[a] -= eps
                bp = edge_basics(ti * S + int(types[j]), dp)
                bm = edge_basics(ti * S + int(types[j]), dm)
                dE[a] = sum(g[b] * (bp[b] - bm[b]) / (2 * eps) for b in range(m.alpha_basic_count))
            f[:, i] += dE
            f[:, j] -= dE
            dx, dy, dz = d
            vir[:, i] -= np.array([dx * dE[0], dy * dE[1], dz * dE[2], dx * dE[1], dx * dE[2],
                                   dy * dE[2], dy * dE[0], dz * dE[0], dz * dE[1]])
    return pe, f, vir
