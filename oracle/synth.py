"""Synthetic receptor writer without the engine library — TEST INFRASTRUCTURE.

A pure-Python restatement of the library's seeded generator
(fastgrid_b200/csrc/synth.cpp, ag_synth_write): the same xoshiro256** stream,
the same self-avoiding chain walk, type repair and charge quantisation, and
the same PDBQT/GPF text, byte for byte (tests/test_host_cpu.py checks that).
It exists so that bench.py's reference arm can write its inputs without
loading libfastgrid_b200.so: the reference arm runs FastGrid's own CPU build
on them and nothing of the engine is mapped into that process.

Every floating-point step is written in the C++ code's order with IEEE double
arithmetic (Python floats), and math.log / math.cos / math.sqrt come from the
same C library, so the coordinates, types and charges are identical.
"""
import math
import os

import numpy as np

_M64 = (1 << 64) - 1
TYPE_NAMES = ("C", "OA", "N", "HD", "A", "SA")
ELEMENTS = ("C", "O", "N", "H", "C", "S")
T_C, T_OA, T_N, T_HD, T_A, T_SA = range(6)


class _Rng:
    """splitmix64 seeding a xoshiro256** generator (synth.cpp Rng)."""

    def __init__(self, seed):
        s = []
        seed &= _M64
        for _ in range(4):
            seed = (seed + 0x9E3779B97F4A7C15) & _M64
            z = seed
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
            s.append(z ^ (z >> 31))
        self.s = s

    @staticmethod
    def _rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & _M64

    def next(self):
        s = self.s
        r = (self._rotl((s[1] * 5) & _M64, 7) * 9) & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = self._rotl(s[3], 45)
        return r

    def uni(self):
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def normal(self):
        u1 = max(self.uni(), 1e-300)
        u2 = self.uni()
        return math.sqrt(-2 * math.log(u1)) * math.cos(2 * math.pi * u2)


def _cround(v):
    """std::round: nearest integer, halves away from zero, sign kept (-0.3 -> -0.0)."""
    t = math.copysign(float(math.trunc(v)), v)
    if abs(v - t) >= 0.5:
        t += math.copysign(1.0, v)
    return t


class _Placer:
    """1.2 A hash grid of placed atoms inside an ellipsoid (synth.cpp Placer)."""

    def __init__(self, semi, origin):
        self.cell = 1.2
        self.ax = [float(a) for a in semi]
        self.o = [float(a) for a in origin]
        self.lo = [self.o[k] - self.ax[k] - 2 * self.cell for k in range(3)]
        self.nc = [int((2 * self.ax[k] + 4 * self.cell) / self.cell) + 1 for k in range(3)]
        self.head = {}
        self.nxt = []
        self.xyz = []

    def inside(self, p):
        s = 0.0
        for k in range(3):
            s += (p[k] - self.o[k]) * (p[k] - self.o[k]) / (self.ax[k] * self.ax[k])
        return s <= 1.0

    def cell_of(self, p):
        return [min(self.nc[k] - 1, max(0, int((p[k] - self.lo[k]) / self.cell))) for k in range(3)]

    def free(self, p):
        c = self.cell_of(p)
        nc = self.nc
        xyz, nxt, head = self.xyz, self.nxt, self.head
        for dz in (-1, 0, 1):
            z = c[2] + dz
            if z < 0 or z >= nc[2]:
                continue
            for dy in (-1, 0, 1):
                y = c[1] + dy
                if y < 0 or y >= nc[1]:
                    continue
                for dx in (-1, 0, 1):
                    x = c[0] + dx
                    if x < 0 or x >= nc[0]:
                        continue
                    a = head.get((z * nc[1] + y) * nc[0] + x, -1)
                    while a >= 0:
                        q = xyz[a]
                        d2 = 0.0
                        d2 += (q[0] - p[0]) * (q[0] - p[0])
                        d2 += (q[1] - p[1]) * (q[1] - p[1])
                        d2 += (q[2] - p[2]) * (q[2] - p[2])
                        if d2 < 1.2 * 1.2:
                            return False
                        a = nxt[a]
        return True

    def add(self, p):
        c = self.cell_of(p)
        ci = (c[2] * self.nc[1] + c[1]) * self.nc[0] + c[0]
        self.nxt.append(self.head.get(ci, -1))
        self.head[ci] = len(self.xyz)
        self.xyz.append((p[0], p[1], p[2]))


def _repair_types(x, t):
    """Retype H-bonding atoms whose bond-vector partners are missing
    (synth.cpp repairTypes); returns the number of changes."""
    n = len(t)
    changed = 0

    def d2(i, j):
        s = 0.0
        for k in range(3):
            s += (x[i][k] - x[j][k]) * (x[i][k] - x[j][k])
        return s

    for ia in range(n):
        lo, hi = max(ia - 20, 0), min(ia + 20, n - 1)
        if t[ia] == T_HD:
            ok = False
            for ib in range(lo, hi + 1):
                if ib != ia and d2(ia, ib) < 1.90:
                    ok = True
                    break
            if not ok:
                t[ia] = T_C
                changed += 1
        elif t[ia] == T_OA or t[ia] == T_SA:
            nbond, i1 = 0, -1
            for ib in range(lo, hi + 1):
                if ib == ia:
                    continue
                r2 = d2(ia, ib)
                is_h = t[ib] == T_HD
                if (r2 < 3.61 and not is_h) or (r2 < 1.69 and is_h):
                    if nbond == 0:
                        i1 = ib
                    nbond += 1
            ok = nbond >= 2
            if nbond == 1:
                for j in range(lo, hi + 1):
                    if j == i1 or j == ia:
                        continue
                    r2 = d2(i1, j)
                    if (r2 < 2.89 and t[j] != T_HD) or (r2 < 1.69 and t[j] == T_HD):
                        ok = True
                        break
            if not ok:
                t[ia] = T_C
                changed += 1
    return changed


def receptor(n_atoms, semi_axes, seed=0, origin=(0.0, 0.0, 0.0), frac=(0.45, 0.18, 0.15, 0.15, 0.05, 0.02),
             charge_sigma=0.2, charge_clip=0.7, net_charge=0.0):
    """(coordinates (n, 3) rounded to 3 decimals, type codes, charges in thousandths)."""
    rng = _Rng(seed)
    pl = _Placer(semi_axes, origin)
    n = n_atoms

    def random_inside():
        for _ in range(100000):
            p = [pl.o[k] + (2 * rng.uni() - 1) * pl.ax[k] for k in range(3)]
            if pl.inside(p) and pl.free(p):
                return p
        return None

    while len(pl.xyz) < n:
        p = random_inside()
        if p is None:
            raise RuntimeError("shape too full for the requested atom count")
        pl.add(p)
        while len(pl.xyz) < n:
            placed = False
            for _ in range(40):
                while True:
                    v = [2 * rng.uni() - 1 for _ in range(3)]
                    nv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
                    if not (nv > 1 or nv < 1e-6):
                        break
                nv = math.sqrt(nv)
                b = 1.22 + 0.13 * rng.uni()
                q = [p[k] + b * v[k] / nv for k in range(3)]
                if pl.inside(q) and pl.free(q):
                    pl.add(q)
                    p = q
                    placed = True
                    break
            if not placed:
                break
    x = [tuple(_cround(v * 1000.0) / 1000.0 for v in a) for a in pl.xyz]

    tot = 0.0
    for f in frac:
        tot += f
    t = []
    for _ in range(n):
        u = rng.uni() * tot
        c = 0.0
        k = 0
        while k < 5:
            c += frac[k]
            if u < c:
                break
            k += 1
        t.append(k)
    for _ in range(8):
        if _repair_types(x, t) == 0:
            break

    q = []
    s = 0.0
    for _ in range(n):
        v = max(-charge_clip, min(charge_clip, rng.normal() * charge_sigma))
        q.append(v)
        s += v
    shift = (net_charge - s) / n
    kq = [int(_cround((v + shift) * 1000.0)) for v in q]
    resid = int(_cround(net_charge * 1000.0)) - sum(kq)
    order = sorted(range(n), key=lambda i: (-abs(kq[i]), i))
    j = 0
    while resid != 0:
        i = order[j % n]
        kq[i] += 1 if resid > 0 else -1
        resid += -1 if resid > 0 else 1
        j += 1
    return np.array(x), t, kq


def write(dirname, stem, n_atoms, semi_axes, npts, ligand_types="A C HD N OA SA", seed=0,
          origin=(0.0, 0.0, 0.0), frac=(0.45, 0.18, 0.15, 0.15, 0.05, 0.02), charge_sigma=0.2, charge_clip=0.7,
          net_charge=0.0, spacing=0.375, dielectric=-0.1465):
    """Write <dir>/<stem>.pdbqt and <stem>.gpf exactly as ag_synth_write does; returns the GPF path."""
    x, t, kq = receptor(n_atoms, semi_axes, seed, origin, frac, charge_sigma, charge_clip, net_charge)
    os.makedirs(dirname, exist_ok=True)
    base = os.path.join(dirname, stem)
    lines = []
    for i in range(n_atoms):
        name = "%s%d" % (ELEMENTS[t[i]], (i % 99) + 1)
        lines.append("ATOM  %5d %-4s %3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f    %6.3f %-2s\n" % (
            (i % 99999) + 1, name, "SYN", "A", (i // 10) % 10000, x[i][0], x[i][1], x[i][2], 1.0, 0.0,
            kq[i] / 1000.0, TYPE_NAMES[t[i]]))
    with open(base + ".pdbqt", "w") as f:
        f.write("".join(lines))
    lig = ligand_types if ligand_types else "A C HD N OA SA"
    g = ["receptor %s.pdbqt\n" % stem, "gridfld %s.maps.fld\n" % stem, "npts %d %d %d\n" % (npts, npts, npts),
         "spacing %.3f\n" % spacing, "gridcenter auto\n", "smooth 0.5\n", "ligand_types %s\n" % lig]
    for tok in lig.replace("\t", " ").split(" "):
        if tok:
            g.append("map %s.%s.map\n" % (stem, tok))
    g += ["elecmap %s.e.map\n" % stem, "dsolvmap %s.d.map\n" % stem, "dielectric %.4f\n" % dielectric]
    with open(base + ".gpf", "w") as f:
        f.write("".join(g))
    return base + ".gpf"
