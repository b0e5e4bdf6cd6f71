"""The FP32 candidate tests of the neighbour fills keep the FP64 list.

The fills classify candidate pairs with FP32 distances and leave only a band
around the cutoff (or everything beyond a coordinate limit) to the FP64 test:

* single box (`k_fill`, engine.cu): FP32 positions relative to their cell's
  corner (FP64 test beyond kRelLimit) plus an FP32 cell-to-cell offset (FP64
  test beyond kOffLimit); in below cutoff2 - m, out above cutoff2 + m, with
  m = 0.01 + 1e-3 cutoff2 A^2;
* batch cells wider than twice the cutoff (`fill_cell_ortho`, batch_fill.cuh):
  FP32 positions relative to the cell's first atom, nearest image by rounding,
  the same band;
* narrower batch cells: a nearest-image pre-test and per-axis image ranges
  with the cutoff widened by 1e-3 A, every survivor taking the FP64 test;
* batch cells with an atom farther than kCompact from the first take the FP64
  scan only.

These tests restate that FP32 arithmetic in numpy (each operation rounded to
FP32; fused multiply-adds with a single rounding) and check, over many pairs
placed near the cutoff at the largest coordinates each path admits, that no
pair within the cutoff is rejected and none beyond it is accepted without the
FP64 test.  The limits are read from the CUDA sources.
"""
import os
import re

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(__file__), "..", "gpumd-sus2-sh_b200", "csrc")
f32 = np.float32


def _const(fname, name):
    text = open(os.path.join(CSRC, fname)).read()
    m = re.search(r"constexpr\s+(?:float|double)\s+" + name + r"\s*=\s*([0-9.]+)f?\s*;", text)
    assert m, name
    return float(m.group(1))


K_REL = _const("engine.cu", "kRelLimit")
K_OFF = _const("engine.cu", "kOffLimit")
K_COMPACT = _const("batch_fill.cuh", "kCompact")


def fma(a, b, c):
    """FP32 fused multiply-add: the FP32 product is exact in FP64, one rounding
    of the FP64 sum (53 bits) then to FP32."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(f32)


def sq3(x, y, z, fused):
    if fused:
        return fma(x, x, fma(y, y, z * z))
    return (x * x + y * y) + z * z


def band(cutoff2):
    m = 0.01 + 1e-3 * cutoff2
    return f32(cutoff2 - m), f32(cutoff2 + m)


def unit(rng, n):
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1, keepdims=True)


def near_cutoff(rng, n, cutoff2, spread):
    """Distances within +-spread (A^2, in r^2) of the cutoff, denser at it."""
    return np.sqrt(cutoff2 + spread * rng.uniform(-1.0, 1.0, n) ** 3)


@pytest.mark.parametrize("rc", [3.0, 6.0, 10.5])
@pytest.mark.parametrize("fused", [False, True])
def test_single_box_fill_classification(rc, fused):
    rng = np.random.default_rng(int(rc * 10) + fused)
    cutoff2 = rc * rc
    lo, hi = band(cutoff2)
    n = 400_000
    # home-relative positions of i and of the candidate up to the FP32 limit;
    # the cell offset is whatever places the pair at the sampled distance
    P = rng.uniform(-K_REL, K_REL, (n, 3))
    Q = rng.uniform(-K_REL, K_REL, (n, 3))
    d = unit(rng, n) * near_cutoff(rng, n, cutoff2, 4 * (0.01 + 1e-3 * cutoff2))[:, None]
    O = d - Q + P
    assert np.abs(O).max() <= K_OFF
    fx = O.astype(f32) - P.astype(f32)
    dx = Q.astype(f32) + fx
    d2 = sq3(dx[:, 0], dx[:, 1], dx[:, 2], fused)
    true2 = ((Q + O) - P) ** 2
    inside = true2.sum(axis=1) < cutoff2
    assert inside.any() and (~inside).any()
    assert np.all(d2[inside] < hi), "a pair within the cutoff is rejected"
    assert np.all(inside[d2 <= lo]), "a pair beyond the cutoff is accepted without the FP64 test"


def _wrapped_pairs(rng, n, L, periodic, cutoff2, spread):
    """Atom pairs of one cell near the cutoff: absolute positions wrapped into
    [0, L) along periodic axes (open axes up to the compact limit), and the
    first atom of the cell."""
    o = np.where(periodic, rng.uniform(0, 1, (n, 3)) * L, 0.0)
    pi = np.where(periodic, rng.uniform(0, 1, (n, 3)) * L, rng.uniform(-K_COMPACT, K_COMPACT, (n, 3)))
    d = unit(rng, n) * near_cutoff(rng, n, cutoff2, spread)[:, None]
    pj = pi + d
    pj = np.where(periodic, pj - np.floor(pj / L) * L, pj)
    keep = (np.abs(pi - o) <= K_COMPACT).all(axis=1) & (np.abs(pj - o) <= K_COMPACT).all(axis=1)
    return keep, o[keep], pi[keep], pj[keep]


@pytest.mark.parametrize("rc", [5.0, 8.0])
def test_wide_batch_cell_classification(rc):
    rng = np.random.default_rng(int(rc))
    cutoff2 = rc * rc
    cutm = f32(np.sqrt(cutoff2)) + f32(1e-3)
    lo2, hi2 = band(cutoff2)
    n = 300_000
    # edges from just above twice the widened cutoff to beyond the compact limit
    L = np.exp(rng.uniform(np.log(2 * float(cutm) * 1.0001), np.log(3 * K_COMPACT), (n, 3)))
    periodic = rng.uniform(size=(n, 3)) < 0.8
    keep, o, pi, pj = _wrapped_pairs(rng, n, L, periodic, cutoff2, 4 * (0.01 + 1e-3 * cutoff2))
    L, periodic = L[keep], periodic[keep]
    assert len(o) > n // 4
    Lf = L.astype(f32)
    jx = np.where(periodic, f32(1.0) / Lf, f32(0.0))
    fi = (pi - o).astype(f32)
    fj = (pj - o).astype(f32)
    dx = fj - fi
    t = np.rint((dx * jx).astype(f32))
    e = fma(-t, Lf, dx)
    m2 = fma(e[:, 0], e[:, 0], fma(e[:, 1], e[:, 1], e[:, 2] * e[:, 2]))
    # exact nearest image in FP64 (unique within the cutoff: L > 2 rc)
    dd = pj - pi
    k = np.where(periodic, np.rint(dd / L), 0.0)
    true2 = ((dd - k * L) ** 2).sum(axis=1)
    inside = true2 < cutoff2
    assert inside.any() and (~inside).any()
    assert np.all(m2[inside] < hi2), "a pair within the cutoff is rejected"
    assert np.all(t[inside] == k[inside]), "the nearest image is missed"
    assert np.all(inside[m2 <= lo2]), "a pair beyond the cutoff is accepted without the FP64 test"


def _narrow_survivors(fi, fj, L, r, cutm, fused=True):
    """Images (tx, ty, tz) of each pair that the narrow-cell scan hands to the
    FP64 test: the nearest-image pre-test, the per-axis image ranges and the
    per-axis partial sums, all in FP32.  Returns a set per pair."""
    cutm2 = f32(cutm * cutm)
    Lf = L.astype(f32)
    iL = f32(1.0) / Lf
    d = fj - fi
    m2 = np.zeros(len(d), dtype=f32)
    for a in range(3):
        t = np.where(r[:, a] > 0, np.rint((d[:, a] * iL[:, a]).astype(f32)), f32(0.0)).astype(f32)
        e = fma(-t, Lf[:, a], d[:, a]) if fused else (d[:, a] - t * Lf[:, a]).astype(f32)
        m2 = fma(e, e, m2) if fused else (m2 + e * e).astype(f32)
    near = m2 < cutm2
    lo = np.maximum(-r, np.ceil(((-cutm - d) * iL).astype(f32)).astype(int))
    hi = np.minimum(r, np.floor(((cutm - d) * iL).astype(f32)).astype(int))
    out = []
    for p in range(len(d)):
        s = set()
        if near[p]:
            for tz in range(lo[p, 2], hi[p, 2] + 1):
                ez = fma(np.array([tz], f32), Lf[p, 2:3], d[p, 2:3])[0]
                ez2 = f32(ez * ez)
                if ez2 >= cutm2:
                    continue
                for ty in range(lo[p, 1], hi[p, 1] + 1):
                    ey = fma(np.array([ty], f32), Lf[p, 1:2], d[p, 1:2])[0]
                    eyz2 = fma(np.array([ey]), np.array([ey]), np.array([ez2]))[0]
                    if eyz2 >= cutm2:
                        continue
                    for tx in range(lo[p, 0], hi[p, 0] + 1):
                        ex = fma(np.array([tx], f32), Lf[p, 0:1], d[p, 0:1])[0]
                        if fma(np.array([ex]), np.array([ex]), np.array([eyz2]))[0] >= cutm2:
                            continue
                        s.add((tx, ty, tz))
        out.append(s)
    return out


def _narrow_case(rng, n, rc, coord_scale):
    """Pairs in cells with one or two edges shorter than twice the cutoff (reach
    1 or 2) and the others up to coord_scale, near the cutoff for one image."""
    cutoff2 = rc * rc
    short = rng.uniform(0.55 * rc, 2.0 * rc, (n, 3))
    long_ = rng.uniform(2.0 * rc, coord_scale, (n, 3))
    L = np.where(rng.uniform(size=(n, 3)) < 0.5, short, long_)
    L[:, 0] = short[:, 0]  # at least one narrow periodic edge
    r = np.minimum(2, np.maximum(1, np.ceil(rc / L - 1e-12))).astype(int)
    pi = rng.uniform(0, 1, (n, 3)) * L
    img = rng.integers(-1, 2, (n, 3)) * (r > 0)
    d = unit(rng, n) * near_cutoff(rng, n, cutoff2, 0.02)[:, None]
    pj = pi + d - img * L
    pj = pj - np.floor(pj / L) * L
    o = rng.uniform(0, 1, (n, 3)) * L
    return L, r, o, pi, pj


@pytest.mark.parametrize("rc", [5.0, 7.0])
@pytest.mark.parametrize("fused", [True, False])
def test_narrow_batch_cell_keeps_every_image_within_the_cutoff(rc, fused):
    rng = np.random.default_rng(100 + int(rc))
    cutoff2 = rc * rc
    cutm = f32(np.sqrt(cutoff2)) + f32(1e-3)
    L, r, o, pi, pj = _narrow_case(rng, 3000, rc, 2 * K_COMPACT)
    keep = (np.abs(pi - o) <= K_COMPACT).all(axis=1) & (np.abs(pj - o) <= K_COMPACT).all(axis=1)
    L, r, o, pi, pj = L[keep], r[keep], o[keep], pi[keep], pj[keep]
    fi, fj = (pi - o).astype(f32), (pj - o).astype(f32)
    surv = _narrow_survivors(fi, fj, L, r, cutm, fused)
    dd = pj - pi
    checked = 0
    for p in range(len(dd)):
        for tz in range(-r[p, 2], r[p, 2] + 1):
            for ty in range(-r[p, 1], r[p, 1] + 1):
                for tx in range(-r[p, 0], r[p, 0] + 1):
                    t = np.array([tx, ty, tz])
                    if (((dd[p] + t * L[p]) ** 2).sum()) < cutoff2:
                        checked += 1
                        assert (tx, ty, tz) in surv[p], (p, tx, ty, tz)
    assert checked > 1000


def _narrow_pre_test_error(rng, n, scale, rc=6.0):
    """Largest error (A) of the narrow path's FP32 nearest-image distance for
    pairs at the cutoff in a 7.6 x 7.6 A wire of length scale..2 scale, the
    pair and the cell's first atom up to scale apart along the wire."""
    L = np.column_stack([np.full(n, 7.6), np.full(n, 7.6), rng.uniform(scale, 2 * scale, n)])
    pi = rng.uniform(0, 1, (n, 3)) * L
    u = unit(rng, n)
    u[:, 2] *= 4
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pj = pi + u * rc
    pj = pj - np.floor(pj / L) * L
    o = np.zeros((n, 3))
    o[:, 2] = np.where(pi[:, 2] > 0.5 * L[:, 2], 0.0, L[:, 2] - 1e-3)
    keep = (np.abs(pi - o).max(axis=1) <= 2 * scale) & (np.abs(pj - o).max(axis=1) <= 2 * scale)
    fi, fj = (pi - o).astype(f32), (pj - o).astype(f32)
    Lf = L.astype(f32)
    d = fj - fi
    t = np.rint((d * (f32(1.0) / Lf)).astype(f32)).astype(f32)
    e = fma(-t, Lf, d)
    m2 = fma(e[:, 0], e[:, 0], fma(e[:, 1], e[:, 1], e[:, 2] * e[:, 2]))
    D = pj - pi
    true = np.sqrt(((D - np.rint(D / L) * L) ** 2).sum(axis=1))
    return np.abs(np.sqrt(m2.astype(np.float64)) - true)[keep].max()


def test_compact_limit_keeps_the_narrow_pre_test_within_its_margin():
    # the narrow path widens the cutoff by 1e-3 A: at the compact limit its
    # FP32 distances are within a quarter of that; at 16,000-32,000 A (cells
    # that now take the FP64 scan) the error passes the margin
    rng = np.random.default_rng(7)
    assert _narrow_pre_test_error(rng, 200_000, K_COMPACT / 2) < 0.25e-3
    assert _narrow_pre_test_error(rng, 200_000, 16384.0) > 1e-3
