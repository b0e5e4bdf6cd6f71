"""Oracle (test infrastructure only): FP64 CPU restatement of the SUS2-SH real
Clebsch-Gordan standard product graph and of the SUS2-SH ``.mtp`` reader.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; it is the checker, never the product.  The product
path is the CUDA library under ``gpumd-sus2-sh_b200/csrc``.

Every function restates the reference algorithm of hu-yanxiao/GPUMD-SUS2-SH and
cites the ``src/force/sus2_sh.cu`` lines it follows.  Parity of this module is
pinned by the graph-count known answers the reference's design notes publish
(``docs/gpumd-sus2-sh-interface-plan.md:24-40,346-355,629-630,990-995,1049``);
see ``tests/test_oracle_graph.py``.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field
from functools import lru_cache

# ---------------------------------------------------------------------------
# Clebsch-Gordan and the real/complex spherical-harmonic map
# ---------------------------------------------------------------------------


def _fact(n: int) -> float:
    """n! as a double, 0 for n < 0 (sus2_sh.cu:1090-1100)."""
    if n < 0:
        return 0.0
    v = 1.0
    for i in range(2, n + 1):
        v *= float(i)
    return v


def _triangle(l1: int, l2: int, l3: int) -> bool:
    """Triangle rule |l1-l2| <= l3 <= l1+l2 (sus2_sh.cu:1102-1105)."""
    return abs(l1 - l2) <= l3 <= l1 + l2


def clebsch_gordan(j1: int, m1: int, j2: int, m2: int, j: int, m: int) -> float:
    """Complex-basis CG <j1 m1 j2 m2 | j m> by the Racah sum
    (sus2_sh.cu:1107-1142)."""
    if m != m1 + m2 or not _triangle(j1, j2, j) or abs(m1) > j1 or abs(m2) > j2 or abs(m) > j:
        return 0.0
    pref1 = math.sqrt((2.0 * j + 1.0) * _fact(j1 + j2 - j) * _fact(j1 - j2 + j)
                      * _fact(-j1 + j2 + j) / _fact(j1 + j2 + j + 1))
    pref2 = math.sqrt(_fact(j1 + m1) * _fact(j1 - m1) * _fact(j2 + m2) * _fact(j2 - m2)
                      * _fact(j + m) * _fact(j - m))
    s = 0.0
    for k in range(0, 65):
        a = j1 + j2 - j - k
        b = j1 - m1 - k
        c = j2 + m2 - k
        d = j - j2 + m1 + k
        e = j - j1 - m2 + k
        if a < 0 or b < 0 or c < 0 or d < 0 or e < 0:
            continue
        s += (-1.0 if k % 2 else 1.0) / (_fact(k) * _fact(a) * _fact(b) * _fact(c) * _fact(d) * _fact(e))
    return pref1 * pref2 * s


def _real_from_complex(real_m: int, complex_m: int) -> complex:
    """Unitary real<-complex map entry U[real_m, complex_m] (sus2_sh.cu:1149-1170)."""
    inv = 1.0 / math.sqrt(2.0)
    if real_m == 0:
        return 1.0 + 0j if complex_m == 0 else 0j
    a = abs(real_m)
    if abs(complex_m) != a:
        return 0j
    sign = 1.0 if a % 2 == 0 else -1.0
    if real_m > 0:
        return complex(inv * sign, 0.0) if complex_m == a else complex(inv, 0.0)
    return complex(0.0, -inv * sign) if complex_m == a else complex(0.0, inv)


def _coupling_phase(l1: int, l2: int, L: int) -> complex:
    """i^(l1+l2-L) phase that makes real couplings real (sus2_sh.cu:1172-1184)."""
    return (1 + 0j, 1j, -1 + 0j, -1j)[(l1 + l2 - L) & 3]


@lru_cache(maxsize=None)
def real_cg(l1: int, rm1: int, l2: int, rm2: int, L: int, rM: int) -> float:
    """Real-basis coupling coefficient (sus2_sh.cu:1186-1218).  Cached: the value
    depends only on its arguments, so caching changes no result."""
    s = 0j
    for M in range(-L, L + 1):
        out_u = _real_from_complex(rM, M).conjugate()
        if abs(out_u) == 0.0:
            continue
        for m1 in range(-l1, l1 + 1):
            in1 = _real_from_complex(rm1, m1)
            if abs(in1) == 0.0:
                continue
            for m2 in range(-l2, l2 + 1):
                in2 = _real_from_complex(rm2, m2)
                if abs(in2) == 0.0:
                    continue
                cg = clebsch_gordan(l1, m1, l2, m2, L, M)
                if abs(cg) < 1.0e-14:
                    continue
                s += out_u * cg * in1 * in2
    s *= _coupling_phase(l1, l2, L)
    if abs(s.imag) > 1.0e-10:
        raise ValueError("SUS2_SH standard graph produced a non-real CG coefficient.")
    return s.real


# ---------------------------------------------------------------------------
# Standard graph builder (SHStandardGraphBuilderHost, sus2_sh.cu:1227-1706)
# ---------------------------------------------------------------------------


@dataclass
class Tensor:
    key: str
    l: int
    layer: int
    block: int = -1
    node: list = field(default_factory=list)
    zero: bool = False


@dataclass
class StandardGraph:
    node_count: int
    max_layer: int
    basic: list            # [(k, l, m)] in node order
    products: list         # [(left, right, target, coeff)]
    scalars: list          # scalar node ids, in spec order
    tensor_blocks: list    # [(kind, layer, base, l)]
    cg_blocks: int
    cg_terms: int


class StandardGraphBuilder:
    """Restates SHStandardGraphBuilderHost (sus2_sh.cu:1227-1706)."""

    def __init__(self, lmax: int, kmax: int):
        self.lmax = lmax
        self.kmax = kmax
        self.node_count = 0
        self.q = []                 # (l, k, mu, key) in q-order (sus2_sh.cu:1451-1465)
        self.tensors = []
        self.lookup = {}
        self.product_lookup = {}
        self.products = []          # lists [left, right, target, coeff]
        self.scalars = []
        self.basic = []
        self.tensor_blocks = []
        self.cg_blocks = 0
        self.cg_terms = 0
        self.body_lmax = None

    # sus2_sh.cu:1451-1465: l = lmax..0, k = kmax-1..0
    def _build_q(self):
        for l in range(self.lmax, -1, -1):
            for k in range(self.kmax - 1, -1, -1):
                mu = k * (self.lmax + 1) + l
                self.q.append((l, k, mu, f"q{mu}_l{l}_k{k}"))

    def _add_node(self) -> int:
        n = self.node_count
        self.node_count += 1
        return n

    # sus2_sh.cu:1252-1290
    def _basic_tensor(self, qi: int) -> Tensor:
        l, k, mu, key = self.q[qi]
        if key in self.lookup:
            return self.tensors[self.lookup[key]]
        t = Tensor(key=key, l=l, layer=0)
        for m in range(-l, l + 1):
            t.node.append(self._add_node())
            self.basic.append((k, l, m))
        t.block = len(self.tensor_blocks)
        self.tensor_blocks.append((0, 0, t.node[0], l))
        self.lookup[key] = len(self.tensors)
        self.tensors.append(t)
        return t

    # sus2_sh.cu:1665-1688
    def _add_product(self, left: int, right: int, target: int, coeff: float):
        if abs(coeff) < 1.0e-12:
            return
        if right < left:
            left, right = right, left
        key = (left, right, target)
        idx = self.product_lookup.get(key)
        if idx is not None:
            self.products[idx][3] += coeff
            return
        self.product_lookup[key] = len(self.products)
        self.products.append([left, right, target, coeff])

    # sus2_sh.cu:1292-1449
    def _couple(self, left: Tensor, right: Tensor, L: int) -> Tensor:
        key = f"({left.key}x{right.key})->{L}"
        if key in self.lookup:
            return self.tensors[self.lookup[key]]
        out = Tensor(key=key, l=L, layer=1 + max(left.layer, right.layer))
        if left.zero or right.zero:
            out.zero = True
            self.lookup[key] = len(self.tensors)
            self.tensors.append(out)
            return out
        local = {}        # (lnode, rnode, tcomp) -> coeff, insertion ordered
        logical = {}      # (lcomp, rcomp, tcomp) -> coeff
        for rm1 in range(-left.l, left.l + 1):
            for rm2 in range(-right.l, right.l + 1):
                for rM in range(-L, L + 1):
                    c = real_cg(left.l, rm1, right.l, rm2, L, rM)
                    if abs(c) < 1.0e-12:
                        continue
                    lc, rc, tc = rm1 + left.l, rm2 + right.l, rM + L
                    lk = (lc, rc, tc)
                    logical[lk] = logical.get(lk, 0.0) + c
                    ln, rn = left.node[lc], right.node[rc]
                    if rn < ln:
                        ln, rn = rn, ln
                    pk = (ln, rn, tc)
                    local[pk] = local.get(pk, 0.0) + c
        compact_local = [(k, v) for k, v in local.items() if abs(v) >= 1.0e-12]
        compact_terms = [v for v in logical.values() if abs(v) >= 1.0e-12]
        if not compact_local:
            out.zero = True
            self.lookup[key] = len(self.tensors)
            self.tensors.append(out)
            return out
        for _ in range(2 * L + 1):
            out.node.append(self._add_node())
        out.block = len(self.tensor_blocks)
        self.tensor_blocks.append((1, out.layer, out.node[0], L))
        self.cg_blocks += 1
        self.cg_terms += len(compact_terms)
        self.lookup[key] = len(self.tensors)
        self.tensors.append(out)
        for (ln, rn, tc), c in compact_local:
            self._add_product(ln, rn, out.node[tc], c)
        return out

    def _allowed(self, qi: int, body: int) -> bool:
        return self.q[qi][0] <= self.body_lmax[body]

    # sus2_sh.cu:1472-1494: tuples with non-increasing l and non-increasing k
    def _tuples(self, count: int, body: int):
        out = []
        tup = []

        def rec(pos, max_l, max_k):
            if pos == count:
                out.append(tuple(tup))
                return
            for qi, (l, k, _, _) in enumerate(self.q):
                if not self._allowed(qi, body) or l > max_l or k > max_k:
                    continue
                tup.append(qi)
                rec(pos + 1, l, k)
                tup.pop()

        rec(0, self.lmax, self.kmax - 1)
        return out

    # sus2_sh.cu:1523-1587
    def _collect_specs(self, body_order: int):
        specs = []
        required = [False] * len(self.q)
        L_of = lambda qi: self.q[qi][0]

        def add(body, qs, inter):
            specs.append((body, qs, inter))
            for qi in qs[: body - 1]:
                required[qi] = True

        if body_order >= 2:
            for (a,) in self._tuples(1, 2):
                if L_of(a) == 0:
                    add(2, (a,), 0)
        if body_order >= 3:
            for a, b in self._tuples(2, 3):
                if L_of(a) == L_of(b):
                    add(3, (a, b), 0)
        if body_order >= 4:
            for a, b, c in self._tuples(3, 4):
                l0, l1, l2 = L_of(a), L_of(b), L_of(c)
                if (l0 + l1 + l2) % 2 == 0 and _triangle(l0, l1, l2):
                    add(4, (a, b, c), l2)
        if body_order >= 5:
            for a, b, c, d in self._tuples(4, 5):
                l0, l1, l2, l3 = L_of(a), L_of(b), L_of(c), L_of(d)
                if (l0 + l1 + l2 + l3) % 2 != 0:
                    continue
                lo = max(abs(l0 - l1), abs(l2 - l3))
                hi = min(l0 + l1, l2 + l3)
                for L in range(lo, hi + 1):
                    add(5, (a, b, c, d), L)
        if body_order >= 6:
            for a, b, c, d, e in self._tuples(5, 6):
                l0, l1, l2, l3, l4 = (L_of(a), L_of(b), L_of(c), L_of(d), L_of(e))
                if (l0 + l1 + l2 + l3 + l4) % 2 != 0:
                    continue
                lo = max(abs(l0 - l1), abs(l2 - l3))
                hi = min(l0 + l1, l2 + l3)
                for L in range(lo, hi + 1):
                    if _triangle(L, l4, L):
                        add(6, (a, b, c, d, e), L)
        return specs, required

    # sus2_sh.cu:1589-1629
    def _build_scalar(self, spec) -> int:
        body, qs, inter = spec
        t0 = self._basic_tensor(qs[0])
        if body == 2:
            return t0.node[0]
        t1 = self._basic_tensor(qs[1])
        if body == 3:
            s = self._couple(t0, t1, 0)
            return -1 if s.zero else s.node[0]
        t2 = self._basic_tensor(qs[2])
        if body == 4:
            pair = self._couple(t0, t1, inter)
            if pair.zero:
                return -1
            s = self._couple(pair, t2, 0)
            return -1 if s.zero else s.node[0]
        t3 = self._basic_tensor(qs[3])
        left = self._couple(t0, t1, inter)
        right_pair = self._couple(t2, t3, inter)
        if body == 6:
            t4 = self._basic_tensor(qs[4])
            if left.zero or right_pair.zero:
                return -1
            right = self._couple(right_pair, t4, inter)
            if right.zero:
                return -1
            s = self._couple(left, right, 0)
            return -1 if s.zero else s.node[0]
        if left.zero or right_pair.zero:
            return -1
        s = self._couple(left, right_pair, 0)
        return -1 if s.zero else s.node[0]

    def build(self, body_order: int, body_lmax) -> StandardGraph:
        """BuildGraph + AddScalars (sus2_sh.cu:1231-1249,1643-1658)."""
        self.body_lmax = list(body_lmax)
        self._build_q()
        specs, required = self._collect_specs(body_order)
        for qi in range(len(self.q)):
            if required[qi]:
                self._basic_tensor(qi)
        for spec in specs:
            s = self._build_scalar(spec)
            if s >= 0:
                self.scalars.append(s)
        prods = [tuple(p) for p in self.products if abs(p[3]) >= 1.0e-12]
        max_layer = max((tb[1] for tb in self.tensor_blocks), default=0)
        return StandardGraph(self.node_count, max_layer, list(self.basic), prods,
                             list(self.scalars), list(self.tensor_blocks),
                             self.cg_blocks, self.cg_terms)


def build_standard_graph(lmax: int, kmax: int, body_order: int, body_lmax=None) -> StandardGraph:
    """Convenience wrapper; ``body_lmax`` is indexed by body order (length 7),
    defaulting to ``lmax`` everywhere as the reader does (sus2_sh.cu:2289)."""
    if body_lmax is None:
        body_lmax = [lmax] * 7
    return StandardGraphBuilder(lmax, kmax).build(body_order, body_lmax)


def body_lmax_from_list(lmax: int, body_order: int, values) -> list:
    """sh_body_l_max = {a,b,c,d[,e]} -> per-body-order table (sus2_sh.cu:2289-2305)."""
    table = [lmax] * 7
    for body in range(2, 2 + len(values)):
        table[body] = values[body - 2]
    return table


# ---------------------------------------------------------------------------
# Explicit row / back-row metadata (build_explicit_sh_graph_metadata,
# sus2_sh.cu:1913-2093) and the terminal-scalar classification of the
# constructor (sus2_sh.cu:8149-8196).
# ---------------------------------------------------------------------------


def explicit_metadata(node_count: int, basic_count: int, products, mapping):
    """Returns dict with rows [(layer, target, [(l, r, c)])], back rows
    [(layer, source, [(target, other, c)])], max_layer and terminal flags."""
    terms_by_target = [[] for _ in range(node_count)]
    last_def = [-1] * node_count
    for p, (l, r, t, c) in enumerate(products):
        if not (0 <= l < node_count and 0 <= r < node_count and 0 <= t < node_count):
            raise ValueError("SUS2_SH explicit product graph index out of range.")
        if t < basic_count:
            raise ValueError("SUS2_SH explicit product graph writes into a basic moment.")
        terms_by_target[t].append((l, r, c))
        last_def[t] = p
    for p, (l, r, t, c) in enumerate(products):
        for s in (l, r):
            if s >= basic_count and last_def[s] < 0:
                raise ValueError("SUS2_SH explicit product graph references an undefined moment.")
            if s >= basic_count and last_def[s] >= p:
                raise ValueError("SUS2_SH explicit product graph is not topologically ordered.")
    defined = [i < basic_count for i in range(node_count)]
    targets = [t for t in range(basic_count, node_count) if terms_by_target[t]]
    for t in targets:
        defined[t] = True
    targets.sort(key=lambda t: (last_def[t], t))
    for m in mapping:
        if m < 0 or m >= node_count or not defined[m]:
            raise ValueError("SUS2_SH alpha_moment_mapping references an undefined moment.")
    node_layer = [0] * node_count
    max_layer = 0
    for t in targets:
        src = 0
        for l, r, _ in terms_by_target[t]:
            src = max(src, node_layer[l], node_layer[r])
        node_layer[t] = src + 1
        max_layer = max(max_layer, src + 1)
    rows = []
    for layer in range(1, max_layer + 1):
        for t in sorted(x for x in targets if node_layer[x] == layer):
            rows.append((layer, t, list(terms_by_target[t])))
    back = []
    for layer in range(1, max_layer + 1):
        by_src = {}
        for (lay, t, terms) in rows:
            if lay != layer:
                continue
            for l, r, c in terms:
                by_src.setdefault(l, []).append((t, r, c))
                by_src.setdefault(r, []).append((t, l, c))
        for s in sorted(by_src):
            back.append((layer, s, by_src[s]))
    used = [False] * node_count
    for (_, _, terms) in rows:
        for l, r, _ in terms:
            used[l] = used[r] = True
    scalar_of = {}
    for s, m in enumerate(mapping):
        scalar_of[m] = s
    terminal = [False] * node_count
    for (_, t, _) in rows:
        if t in scalar_of and not used[t]:
            terminal[t] = True
    return {"rows": rows, "back": back, "max_layer": max_layer, "terminal": terminal,
            "node_layer": node_layer}


# ---------------------------------------------------------------------------
# .mtp reader (load_sh_model, sus2_sh.cu:2105-2482; text helpers :275-477)
# ---------------------------------------------------------------------------


class MtpError(ValueError):
    pass


def _after(text: str, token: str) -> str:
    pos = text.find(token)
    if pos < 0:
        raise MtpError("Missing token in SUS2-SH model file: " + token)
    pos += len(token)
    end = text.find("\n", pos)
    return (text[pos:] if end < 0 else text[pos:end]).strip()


def _braced(text: str, token: str) -> str:
    pos = text.find(token)
    if pos < 0:
        raise MtpError("Missing token in SUS2-SH model file: " + token)
    pos = text.find("{", pos)
    if pos < 0:
        raise MtpError("Missing token in SUS2-SH model file: {")
    depth = 0
    start = pos
    for i in range(pos, len(text)):
        if text[i] == "{":
            if depth == 0:
                start = i
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start:i + 1]
    raise MtpError("Unterminated braced section in SUS2-SH model file: " + token)


def _top_groups(text: str):
    groups, depth, start = [], 0, 0
    for i, ch in enumerate(text):
        if ch == "{":
            if depth == 1:
                start = i
            depth += 1
        elif ch == "}":
            if depth == 2:
                groups.append(text[start:i + 1])
            depth -= 1
    return groups


def _all_groups(text: str):
    groups, depth, start = [], 0, 0
    for i, ch in enumerate(text):
        if ch == "{":
            if depth == 0:
                start = i
            depth += 1
        elif ch == "}":
            depth -= 1
            if depth == 0:
                groups.append(text[start:i + 1])
    return groups


_num_re = re.compile(r"[{},]")


def _numbers(text: str, kind=float):
    """parse_numbers: braces and commas become spaces, then read numbers until
    the first token that does not parse (sus2_sh.cu:443-477)."""
    out = []
    for tok in _num_re.sub(" ", text).split():
        try:
            out.append(kind(tok) if kind is float else int(tok))
        except ValueError:
            break
    return out


@dataclass
class MtpModel:
    species_count: int
    sh_l_max: int
    sh_k_max: int
    sh_body_order: int
    radial_basis_type: str
    rational: bool
    max_dist: float
    rb_size: int
    radial_funcs_count: int
    alpha_moments_count: int
    alpha_basic_count: int
    alpha_scalar_moments: int
    scaling: float
    body_lmax: list
    shift_coeffs: list
    scal_coeffs: list
    species_coeffs: list
    moment_coeffs: list
    alpha_moment_mapping: list
    alpha_basic: list        # [(mu, l, m)]
    products: list           # [(l, r, t, c)]
    radial_coeffs: list      # [Kmu * rb]
    radial_type_coeffs: list # [S]
    # ZBL short-range term (load_sh_model, sus2_sh.cu:2132-2147)
    zbl_enabled: bool = False
    zbl_inner: float = 0.7
    zbl_outer: float = 1.4
    zbl_typewise: bool = False
    zbl_typewise_factor: float = 0.7
    zbl_atomic_numbers: list = None
    # body order of each scalar (sh_scalar_info, sus2_sh.cu:2354-2378)
    scalar_body: list = None
    # two-layer mu-body gate (sus2_sh.cu:2153-2268, metadata :2412-2478)
    gate: dict = None
    # RBLaguerre_log1p[_lmp] radial basis (sus2_sh.cu:363-374,3299-3352)
    laguerre: bool = False


def load_mtp(path: str) -> MtpModel:
    """Restates load_sh_model (sus2_sh.cu:2105-2482) for the non-gate models
    the engine targets, ZBL metadata included (:2132-2147).  ``RBChebyshev_sss_rational`` is accepted as the
    rational map the reference documents (README.md:45,55-56)."""
    with open(path) as fh:
        text = fh.read()
    if _after(text, "version =") != "1.1.0":
        raise MtpError("SUS2_SH currently supports only version = 1.1.0.")
    if _after(text, "potential_tag =") != "SUS2-SH":
        raise MtpError("SUS2_SH selected for a non-SUS2-SH model.")
    scaling = float(_after(text, "scaling ="))
    scaling_map = _after(text, "scaling_map =")
    S = int(_after(text, "species_count ="))
    L = int(_after(text, "sh_l_max ="))
    K = int(_after(text, "sh_k_max ="))
    body = int(_after(text, "sh_body_order ="))
    if "sh_parity =" in text and _after(text, "sh_parity =") != "even":
        raise MtpError("SUS2_SH GPUMD backend currently supports even parity models only.")
    rtype = _after(text, "radial_basis_type =")
    laguerre = False
    if rtype in ("RBChebyshev_sss", "RBChebyshev_sss_lmp"):
        rational = False
    elif rtype in ("RBLaguerre_log1p", "RBLaguerre_log1p_lmp"):
        rational, laguerre = False, True
    elif rtype in ("RBChebyshev_sss_rational", "RBChebyshev_sss_rational_lmp"):
        rational = True
    else:
        raise MtpError("Unsupported SUS2_SH radial_basis_type: " + rtype)
    max_dist = float(_after(text, "max_dist ="))
    rb = int(_after(text, "radial_basis_size ="))
    kmu = int(_after(text, "radial_funcs_count ="))
    M = int(_after(text, "alpha_moments_count ="))
    Bb = int(_after(text, "alpha_index_basic_count ="))
    nsc = int(_after(text, "alpha_scalar_moments ="))
    if scaling_map != "LK":
        raise MtpError("SUS2_SH requires scaling_map = LK.")
    if L < 0 or L > 6:
        raise MtpError("SUS2_SH supports sh_l_max in [0,6].")
    if body < 2 or body > 6:
        raise MtpError("SUS2_SH supports sh_body_order in [2,6].")
    if K <= 0 or kmu != K * (L + 1):
        raise MtpError("SUS2_SH inconsistent sh_k_max/radial_funcs_count.")
    if rb <= 0 or rb > 16 or kmu > 48:
        raise MtpError("SUS2_SH GPU scratch limit exceeded: rb_size<=16, radial_funcs_count<=48.")
    if Bb <= 0 or Bb > 320:
        raise MtpError("SUS2_SH GPU scratch limit exceeded: alpha_index_basic_count<=320.")
    blmax = [L] * 7
    if "sh_body_l_max =" in text:
        vals = _numbers(_braced(text, "sh_body_l_max ="), int)
        expected = 5 if body >= 6 else 4
        if len(vals) != expected:
            raise MtpError("Unexpected SUS2_SH sh_body_l_max size.")
        for b in range(2, 2 + expected):
            blmax[b] = vals[b - 2]
    for b in range(2, body + 1):
        if blmax[b] < 0 or blmax[b] > L:
            raise MtpError("SUS2_SH sh_body_l_max entry is out of range.")
    shift = _numbers(_braced(text, "shift_coeffs ="))
    scal = _numbers(_braced(text, "scal_coeffs ="))
    species = _numbers(_braced(text, "species_coeffs ="))
    moment = _numbers(_braced(text, "moment_coeffs ="))
    mapping = _numbers(_braced(text, "alpha_moment_mapping ="), int)
    raw = _numbers(_braced(text, "alpha_index_basic ="), int)
    if len(raw) != 3 * Bb:
        raise MtpError("Unexpected SUS2_SH alpha_index_basic size.")
    basic = []
    for i in range(Bb):
        k, l, m = raw[3 * i: 3 * i + 3]
        if k < 0 or k >= K or l < 0 or l > L or abs(m) > l:
            raise MtpError("Invalid SUS2_SH alpha_index_basic entry.")
        basic.append((k * (L + 1) + l, l, m))
    P = int(_after(text, "sh_product_count ="))
    groups = _top_groups(_braced(text, "sh_products ="))
    if len(groups) != P:
        raise MtpError("Unexpected SUS2_SH sh_products size.")
    prods = []
    for g in groups:
        v = _numbers(g)
        if len(v) != 4:
            raise MtpError("Invalid SUS2_SH product entry.")
        l, r, t = int(v[0]), int(v[1]), int(v[2])
        if not (0 <= l < M and 0 <= r < M and 0 <= t < M):
            raise MtpError("SUS2_SH product index out of range.")
        prods.append((l, r, t, v[3]))
    rstart = text.find("radial_coeffs")
    if rstart < 0:
        raise MtpError("Missing token in SUS2-SH model file: radial_coeffs")
    rend = text.find("alpha_moments_count", rstart)
    if rend < 0:
        raise MtpError("Missing token in SUS2-SH model file: alpha_moments_count")
    rgroups = _all_groups(text[rstart:rend])
    if len(rgroups) < kmu:
        raise MtpError("Unexpected SUS2_SH radial_coeffs section.")
    radial = [0.0] * (kmu * rb)
    rtc = [1.0] * S
    for mu in range(kmu):
        v = _numbers(rgroups[mu])
        if len(v) != rb + S:
            raise MtpError("Unexpected SUS2_SH radial_coeffs row size.")
        radial[mu * rb: (mu + 1) * rb] = v[:rb]
        if mu == 0:
            rtc = v[rb: rb + S]
    if (len(shift) != S or len(species) != S or len(scal) != 2 * S * S * kmu
            or len(mapping) != nsc or len(moment) != nsc):
        raise MtpError("Unexpected SUS2_SH coefficient dimensions.")
    # build_explicit_sh_graph_metadata validation (sus2_sh.cu:1913-2006)
    if M <= 0 or Bb <= 0 or Bb > M:
        raise MtpError("SUS2_SH invalid explicit product graph dimensions.")
    try:
        explicit_metadata(M, Bb, prods, mapping)
    except ValueError as exc:
        raise MtpError(str(exc)) from exc
    model = MtpModel(S, L, K, body, rtype, rational, max_dist, rb, kmu, M, Bb, nsc, scaling,
                     blmax, shift, scal, species, moment, mapping, basic, prods, radial, rtc, laguerre=laguerre)
    gate = _parse_gate(text, K, kmu, rb, S) if ("two_layer_gate_enabled =" in text
                                                and _bool(_after(text, "two_layer_gate_enabled ="))) else None
    if "sh_scalar_info_count =" in text:
        n = int(_after(text, "sh_scalar_info_count ="))
        if n != nsc:
            raise MtpError("SUS2_SH sh_scalar_info_count should equal alpha_scalar_moments.")
        info = _top_groups(_braced(text, "sh_scalar_info ="))
        if len(info) != n:
            raise MtpError("Unexpected SUS2_SH sh_scalar_info size.")
        model.scalar_body = []
        for g in info:
            v = _numbers(g, int)
            if not v:
                raise MtpError("Invalid SUS2_SH sh_scalar_info entry.")
            if v[0] < 2 or v[0] > body:
                raise MtpError("SUS2_SH sh_scalar_info body order is out of range.")
            model.scalar_body.append(v[0])
    elif gate is not None:
        raise MtpError("GPUMD SUS2_SH mu-body gate requires sh_scalar_info metadata.")
    if gate is not None:
        _gate_metadata(model, gate)
        model.gate = gate
    if "zbl_enabled =" in text and _bool(_after(text, "zbl_enabled =")):
        model.zbl_enabled = True
        if "zbl_inner =" in text:
            model.zbl_inner = float(_after(text, "zbl_inner ="))
        if "zbl_outer =" in text:
            model.zbl_outer = float(_after(text, "zbl_outer ="))
        if "zbl_typewise_cutoff_enabled =" in text:
            model.zbl_typewise = _bool(_after(text, "zbl_typewise_cutoff_enabled ="))
        else:
            model.zbl_typewise = "zbl_typewise_cutoff_factor =" in text
        if "zbl_typewise_cutoff_factor =" in text:
            model.zbl_typewise_factor = float(_after(text, "zbl_typewise_cutoff_factor ="))
        if "zbl_atomic_numbers =" in text:
            model.zbl_atomic_numbers = _numbers(_braced(text, "zbl_atomic_numbers ="), int)
    return model


def _parse_gate(text: str, K: int, kmu: int, rb: int, S: int) -> dict:
    """The gate keys of load_sh_model (sus2_sh.cu:2153-2268), same checks and
    messages; neighbour site mode and shared-radial tables only."""
    mode = _after(text, "two_layer_gate_mode =") if "two_layer_gate_mode =" in text else "legacy"
    if mode == "mu-body-linear-combo":
        mode_id = 1
    elif mode in ("mu-scalar-full", "mu-body-order"):
        mode_id = 2
    elif mode == "legacy":
        raise MtpError("GPUMD SUS2_SH mu-body-order branch requires two_layer_gate_mode = "
                       "mu-body-linear-combo or mu-scalar-full; legacy gate models are not supported here.")
    else:
        raise MtpError("Unsupported SUS2_SH two_layer_gate_mode in GPUMD: " + mode)
    if "two_layer_gate_include_one_body =" in text and _bool(_after(text, "two_layer_gate_include_one_body =")):
        raise MtpError("GPUMD SUS2_SH gate backend requires two_layer_gate_include_one_body = false.")
    if "two_layer_gate_scale_mode =" in text:
        raise MtpError("GPUMD SUS2_SH mu-body gate does not support two_layer_gate_scale_mode.")
    if "two_layer_gate_bias =" in text:
        raise MtpError("GPUMD SUS2_SH mu-body gate does not support two_layer_gate_bias.")
    if "two_layer_residual_enabled =" in text and _bool(_after(text, "two_layer_residual_enabled =")):
        raise MtpError("GPUMD SUS2_SH mu-body gate does not support residual gate fields.")
    if "two_layer_gate_site_mode =" in text:
        site = _after(text, "two_layer_gate_site_mode =")
        if site == "double":
            raise MtpError("GPUMD SUS2_SH mu-body gate currently supports two_layer_gate_site_mode = neighbor. "
                           "Double-site gate will be added after the single-gate CUDA path is verified.")
        if site != "neighbor":
            raise MtpError("Unsupported SUS2_SH two_layer_gate_site_mode in GPUMD: " + site)
    amp = float(_after(text, "two_layer_gate_tanh_amplitude =")) if "two_layer_gate_tanh_amplitude =" in text else 0.8
    if not math.isfinite(amp) or amp < 0.0 or amp > 1.0:
        raise MtpError("SUS2_SH two_layer_gate_tanh_amplitude should be finite and in [0,1].")
    radial_mode = _after(text, "two_layer_gate_radial_mode =") if "two_layer_gate_radial_mode =" in text else ""
    if radial_mode != "shared-radial":
        raise MtpError("GPUMD SUS2_SH gate backend currently requires shared-radial gate mode.")
    if int(_after(text, "two_layer_gate_body_order_max =")) != K + 1:
        raise MtpError("SUS2_SH two_layer_gate_body_order_max should equal sh_k_max + 1.")
    nbody = K
    nrad = int(_after(text, "two_layer_gate_radial_coeff_count ="))
    if nrad != kmu * rb:
        raise MtpError("SUS2_SH two-layer gate radial coefficient count is inconsistent.")
    radial = _numbers(_braced(text, "two_layer_gate_radial_coeffs ="))
    if len(radial) != nrad:
        raise MtpError("SUS2_SH two-layer gate radial coeff list has wrong size.")
    if "two_layer_gate_additive_coeff_count =" in text:
        if int(_after(text, "two_layer_gate_additive_coeff_count =")) != S:
            raise MtpError("SUS2_SH two-layer gate additive coefficient count is inconsistent.")
        additive = _numbers(_braced(text, "two_layer_gate_additive_coeffs ="))
        if len(additive) != S:
            raise MtpError("SUS2_SH two-layer gate additive coeff list has wrong size.")
    else:
        additive = [1.0] * S
    nw = int(_after(text, "two_layer_gate_weight_count ="))
    if nw <= 0:
        raise MtpError("SUS2_SH two-layer gate should contain at least one scalar weight.")
    qidx = _numbers(_braced(text, "two_layer_gate_scalar_indices ="), int)
    weights = _numbers(_braced(text, "two_layer_gate_weights ="))
    if not qidx:
        raise MtpError("SUS2_SH two-layer gate scalar index list is empty.")
    expected = kmu * len(qidx) if mode_id == 2 else len(qidx)
    if nw != expected or len(weights) != expected:
        raise MtpError("SUS2_SH two-layer gate scalar index/weight dimensions are inconsistent.")
    mix = []
    if mode_id == 1:
        nmix = int(_after(text, "two_layer_gate_body_mix_weight_count ="))
        if nmix != kmu * nbody:
            raise MtpError("SUS2_SH two-layer gate body-mix weight count is inconsistent.")
        mix = _numbers(_braced(text, "two_layer_gate_body_mix_weights ="))
        if len(mix) != nmix:
            raise MtpError("SUS2_SH two-layer gate body-mix weight list has wrong size.")
    elif "two_layer_gate_body_mix_weights =" in text or "two_layer_gate_body_mix_weight_count =" in text:
        raise MtpError("SUS2_SH mu-scalar-full gate should not contain body-mix weights.")
    return dict(mode=mode_id, amplitude=amp, nbody=nbody, radial=radial, additive=additive,
                scalar_indices=qidx, weights=weights, body_mix=mix)


def _gate_metadata(m: MtpModel, g: dict) -> None:
    """Gate scalar -> moment and body bucket (sus2_sh.cu:2412-2461)."""
    moment_of, body_of = [], []
    present = [False] * g["nbody"]
    for q in g["scalar_indices"]:
        if q < 0 or q >= m.alpha_scalar_moments:
            raise MtpError("SUS2_SH two-layer gate scalar index is out of range.")
        b = m.scalar_body[q] - 2
        if b < 0 or b >= g["nbody"]:
            raise MtpError("SUS2_SH two-layer gate scalar body order is outside the gate range.")
        present[b] = True
        mom = m.alpha_moment_mapping[q]
        if mom < 0 or mom >= m.alpha_moments_count:
            raise MtpError("SUS2_SH two-layer gate mapped moment index is out of range.")
        moment_of.append(mom)
        body_of.append(b)
    if not all(present):
        raise MtpError("SUS2_SH two-layer gate scalar list misses a required body-order bucket.")
    g["moment_of"] = moment_of
    g["body_of"] = body_of


def _bool(token: str) -> bool:
    """parse_optional_bool_after (sus2_sh.cu:343-361): exact tokens."""
    if token in ("1", "true", "TRUE", "yes", "on"):
        return True
    if token in ("0", "false", "FALSE", "no", "off"):
        return False
    raise MtpError("Invalid boolean token in SUS2-SH model file: " + token)


def standard_graph_matches(model: MtpModel, graph: StandardGraph) -> bool:
    """standard_sh_graph_matches (sus2_sh.cu:1872-1911): same counts, same basic
    layout, products equal within 2e-10*(1+|c|), same scalar mapping."""
    if (graph.node_count != model.alpha_moments_count
            or len(graph.basic) != model.alpha_basic_count
            or len(graph.products) != len(model.products)
            or len(graph.scalars) != len(model.alpha_moment_mapping)):
        return False
    L = model.sh_l_max
    for (k, l, m), (mu, ml, mm) in zip(graph.basic, model.alpha_basic):
        if mu != k * (L + 1) + l or ml != l or mm != m:
            return False
    for (el, er, et, ec), (al, ar, at, ac) in zip(graph.products, model.products):
        if al != el or ar != er or at != et or abs(ac - ec) > 2.0e-10 * (1.0 + abs(ec)):
            return False
    return list(graph.scalars) == list(model.alpha_moment_mapping)
