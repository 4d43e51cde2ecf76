"""The tiling schedule of the fused RB-GS sweep (k_rb_sweep, h2_b200/csrc/h2g_sweep.cuh), checked
on the CPU without a GPU: a numpy restatement of the kernel's indexing -- tiles of positions x rows
with one cell of overlap, z chunks, the TMA boxes (x start rounded down to 16 bytes, zero outside
the array), the ring of staged planes, the register windows along z and the colour-0 exchange
buffer -- must reproduce two colour passes bit for bit, write every interior cell exactly once,
never write a guard, and stay inside every shared-memory box.  The tile constants are read from the
kernel's header, so the check follows them.

The per-cell arithmetic is the reference's rbsor_core! update with omega = 1
(src/NonUniform.jl:848-915): separately rounded IEEE double operations in numpy, no FMA.
"""
import itertools
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "h2_b200", "csrc", "h2g_sweep.cuh")


def _const(name):
    m = re.search(rf"constexpr int {name} = ([^;]+);", open(HDR).read())
    return m.group(1)


TPX = int(_const("kSwTPX"))
TJ = int(_const("kSwTJ"))
NS = int(_const("kSwStages"))
RR = 2 * (TJ + 2)
WK = TPX + 32
WX = TPX + 8


class Geo:
    """The colour-split device layout (h2g_internal.cuh)."""

    def __init__(s, MX, MY, MZ):
        s.MX, s.MY, s.MZ = MX, MY, MZ
        s.NX, s.NY, s.NZ = MX - 2, MY - 2, MZ - 2
        half = (MX + 1) // 2
        s.HP = (half + 31) // 32 * 32
        s.HI = (s.NX >> 1) + 1
        s.plane = MY * 2 * s.HP
        s.n = MZ * s.plane

    def row(s, c, j, k):
        return ((k * s.MY + j) * 2 + c) * s.HP

    def off(s, i, j, k):
        return s.row(((i + j + k) & 1) ^ 1, j, k) + (i >> 1)


def align_down(v, a):
    return v - v % a if v >= 0 else -((-v + a - 1) // a) * a


def update(op, k, keys, ci, pp, b, xm, xp, ym, yp, zm, zp):
    k0, kxm, kxp, kym, kyp, kzm, kzp = (int(v) for v in keys)
    P = op["P"]
    bx = (k * P + (k0 & 0x7F)) << 8
    tx, ty, tz = op["tx"], op["ty"], op["tz"]
    cxm, cxp, cym, cyp = tx[bx | kxm], tx[bx | kxp], ty[bx | kym], ty[bx | kyp]
    czm, czp = tz[bx | kzm], tz[(bx + (P << 8)) | kzp]
    s = cxp + cxm
    for t in (cyp, cym, czp, czm):
        s = s + t
    cv = op["conv"][4 * k: 4 * k + 4]
    for t in (0.0 if kxp & 0x80 else cv[1], 0.0 if kxm & 0x80 else cv[0], 0.0 if kyp & 0x80 else cv[3],
              0.0 if kym & 0x80 else cv[2], 0.0 if kzp & 0x80 else op["czp"], 0.0 if kzm & 0x80 else op["czm"]):
        s = s + t
    dd = 0.0 + (s + 0.0)
    ss = cxp * xp
    for c, v in ((cxm, xm), (cyp, yp), (cym, ym), (czp, zp), (czm, zm)):
        ss = ss + c * v
    return pp + 1.0 * ((ss - b) / dd - pp)


def colour_pass(g, op, x, bb, color):
    key, xin, x = op["key"], x, x.copy()
    for k, j, i in itertools.product(range(1, g.NZ + 1), range(1, g.NY + 1), range(1, g.NX + 1)):
        if ((i + j + k) & 1) ^ 1 != color:
            continue
        a = g.off(i, j, k)
        if not key[a] & 0x80:
            continue
        o = [g.off(i - 1, j, k), g.off(i + 1, j, k), g.off(i, j - 1, k), g.off(i, j + 1, k), g.off(i, j, k - 1),
             g.off(i, j, k + 1)]
        x[a] = update(op, k, [key[a]] + [key[q] for q in o], a, xin[a], bb[a], *[xin[q] for q in o])
    return x


def box(g, arr, x0, y0, z, W, H):
    """A TMA box: zero outside the array."""
    out = np.zeros((H, W), dtype=arr.dtype)
    if not 0 <= z < g.MZ:
        return out
    pl = arr[z * g.plane:(z + 1) * g.plane].reshape(2 * g.MY, g.HP)
    ya, yb, xa, xb = max(y0, 0), min(y0 + H, 2 * g.MY), max(x0, 0), min(x0 + W, g.HP)
    if ya < yb and xa < xb:
        out[ya - y0:yb - y0, xa - x0:xb - x0] = pl[ya:yb, xa:xb]
    return out


def fused(g, op, xin, bb, chunks, esize=8):
    A = 16 // esize
    key = op["key"]
    xout = np.zeros(g.n)
    written = np.zeros(g.n, int)
    kc = (g.NZ + chunks - 1) // chunks
    grid = ((g.HI + TPX - 3) // (TPX - 2), (g.NY + TJ - 3) // (TJ - 2), (g.NZ + kc - 1) // kc)
    tx, ty = np.meshgrid(np.arange(TPX), np.arange(TJ))
    for bxi, byi, bzi in itertools.product(*(range(n) for n in grid)):
        q0, r0 = bxi * (TPX - 2) - 1, byi * (TJ - 2)
        kA = 1 + bzi * kc
        kB = min(kA + kc - 1, g.NZ)
        xs, xk, ys = align_down(q0 - 1, A), align_down(q0 - 1, 16), 2 * (r0 - 1)
        assert xs % A == 0 and xk % 16 == 0  # TMA x-coordinate alignment
        first, last = kA - 2, kB + 2
        ring = {}

        def load(pl):
            ring[(pl - first) % NS] = (pl, box(g, xin, xs, ys, pl, WX, RR), box(g, key, xk, ys, pl, WK, RR))

        def X(pl):
            slot = ring[(pl - first) % NS]
            assert slot[0] == pl  # the ring never overwrote a plane still in use
            return slot[1]

        def K(pl):
            slot = ring[(pl - first) % NS]
            assert slot[0] == pl
            return slot[2]

        for pl in range(first, min(first + NS - 2, last) + 1):
            load(pl)
        p, j = q0 + tx, r0 + ty
        cx, ck = p - xs, p - xk
        assert cx.min() >= 1 and cx.max() + 1 < WX and ck.min() >= 1 and ck.max() + 1 < WK
        rr0 = 2 * (ty + 1)
        rr1 = rr0 + 1
        assert (rr1 - 2).min() >= 0 and (rr1 + 2).max() < RR
        owned = (tx >= 1) & (tx < TPX - 1) & (ty >= 1) & (ty < TJ - 1)
        c1v = [None, X(first)[rr1, cx], X(first + 1)[rr1, cx]]
        c1k = [None, K(first)[rr1, ck], K(first + 1)[rr1, ck]]
        c0v, c0k = [None] * 3, [None] * 3
        c0b = {}

        def inside(k, e):
            i = 2 * p + e
            return (j >= 1) & (j <= g.NY) & (p >= 0) & (1 <= k <= g.NZ) & (i >= 1) & (i <= g.NX)

        for s in range(kA - 1, kB + 2):
            if s + 3 <= last:
                load(s + 3)
            c1v = [c1v[1], c1v[2], X(s + 1)[rr1, cx]]
            c1k = [c1k[1], c1k[2], K(s + 1)[rr1, ck]]
            X0, K0 = X(s), K(s)
            # phase A: colour 0 at plane s, tile and overlap
            e = (1 + j + s) & 1
            d = np.where(e == 1, 1, -1)
            pp, k0 = X0[rr0, cx], K0[rr0, ck]
            nv = pp.copy()
            upd = inside(s, e) & ((k0 & 0x80) != 0)
            for a_, b_ in zip(*np.nonzero(upd)):
                xo, ko = X0[rr1[a_, b_], cx[a_, b_] + d[a_, b_]], K0[rr1[a_, b_], ck[a_, b_] + d[a_, b_]]
                own, kown = c1v[1][a_, b_], c1k[1][a_, b_]
                xm, xp = (own, xo) if e[a_, b_] else (xo, own)
                kxm, kxp = (kown, ko) if e[a_, b_] else (ko, kown)
                ci = g.row(0, j[a_, b_], s) + p[a_, b_]
                keys = [k0[a_, b_], kxm, kxp, K0[rr1[a_, b_] - 2, ck[a_, b_]], K0[rr1[a_, b_] + 2, ck[a_, b_]],
                        c1k[0][a_, b_], c1k[2][a_, b_]]
                nv[a_, b_] = update(op, s, keys, ci, pp[a_, b_], bb[ci], xm, xp, X0[rr1[a_, b_] - 2, cx[a_, b_]],
                                    X0[rr1[a_, b_] + 2, cx[a_, b_]], c1v[0][a_, b_], c1v[2][a_, b_])
            c0v = [c0v[1], c0v[2], nv]
            c0k = [c0k[1], c0k[2], k0]
            wr = owned & inside(s, e) & (kA <= s <= kB)
            for a_, b_ in zip(*np.nonzero(wr)):
                ci = g.row(0, j[a_, b_], s) + p[a_, b_]
                xout[ci] = nv[a_, b_]
                written[ci] += 1
            # phase B: colour 1 at plane s-1 (owned), colour-0 neighbours from the previous step
            sb = s - 1
            if sb >= kA:
                Km, C = K(sb), c0b[sb]
                e1 = (j + sb) & 1
                in1 = owned & inside(sb, e1)
                for a_, b_ in zip(*np.nonzero(in1)):
                    pp1, k1 = c1v[0][a_, b_], c1k[0][a_, b_]
                    v = pp1
                    if k1 & 0x80:
                        dd_ = 1 if e1[a_, b_] else -1
                        xo, ko = C[a_, b_ + dd_], Km[rr0[a_, b_], ck[a_, b_] + dd_]
                        own, kown = c0v[1][a_, b_], c0k[1][a_, b_]
                        xm, xp = (own, xo) if e1[a_, b_] else (xo, own)
                        kxm, kxp = (kown, ko) if e1[a_, b_] else (ko, kown)
                        ci = g.row(1, j[a_, b_], sb) + p[a_, b_]
                        keys = [k1, kxm, kxp, Km[rr0[a_, b_] - 2, ck[a_, b_]], Km[rr0[a_, b_] + 2, ck[a_, b_]],
                                c0k[0][a_, b_], c0k[2][a_, b_]]
                        v = update(op, sb, keys, ci, pp1, bb[ci], xm, xp, C[a_ - 1, b_], C[a_ + 1, b_],
                                   c0v[0][a_, b_], c0v[2][a_, b_])
                    ci = g.row(1, j[a_, b_], sb) + p[a_, b_]
                    xout[ci] = v
                    written[ci] += 1
            c0b[s] = nv
    return xout, written


def problem(MX, MY, MZ, seed, P=3):
    g = Geo(MX, MY, MZ)
    rng = np.random.default_rng(seed)
    key = np.zeros(g.n, np.uint8)
    x, bb = np.zeros(g.n), np.zeros(g.n)
    for k, j, i in itertools.product(range(MZ), range(MY), range(MX)):
        a = g.off(i, j, k)
        interior = 1 <= i <= g.NX and 1 <= j <= g.NY and 1 <= k <= g.NZ
        m = interior and rng.random() > 0.03
        key[a] = (0x80 if m else 0) | int(rng.integers(0, P))
        if interior:
            x[a] = rng.standard_normal() if m else 0.0
            bb[a] = rng.standard_normal()
    tabs = {t: rng.uniform(0.5, 2.0, size=(MZ + 1) * P * 256) for t in ("tx", "ty", "tz")}
    op = dict(P=P, key=key, conv=rng.uniform(0.01, 0.1, size=4 * MZ), czm=0.03, czp=0.05, **tabs)
    return g, op, x, bb


# grids: smaller than a tile; several tiles in x and y with z chunks; more chunks than planes; a
# chunk long enough for the ring of staged planes to wrap several times
@pytest.mark.parametrize("MX,MY,MZ,chunks", [(7, 5, 4, 1), (130, 31, 6, 2), (66, 16, 5, 5), (40, 9, 12, 1)])
def test_fused_tiling_reproduces_colour_passes(MX, MY, MZ, chunks):
    g, op, x, bb = problem(MX, MY, MZ, seed=MX + MY)
    ref = colour_pass(g, op, colour_pass(g, op, x, bb, 0), bb, 1)
    out, written = fused(g, op, x, bb, chunks)
    interior = np.zeros(g.n, bool)
    for k, j, i in itertools.product(range(1, g.NZ + 1), range(1, g.NY + 1), range(1, g.NX + 1)):
        interior[g.off(i, j, k)] = True
    assert (written[interior] == 1).all()
    assert not written[~interior].any()
    assert np.array_equal(out[interior], ref[interior])
