"""Generates the golden fixtures of tests/golden/*.json.

The reference (Fortran 77) cannot be compiled here and ships no test
vectors, so these fixtures come from a second, independent restatement of the
reference's arithmetic written in plain Python (IEEE doubles, left-to-right
evaluation, no fused multiply-add -- the same rounding as gfortran -O2 on
x86-64), on small hand-built configurations whose answers are also checked
analytically where an analytic answer exists (LJ minimum, zero crossing,
inclusive cut-offs, clusters built by construction).  The C oracle must
reproduce every number bit for bit; floats are stored as hex strings.

Run:  python tests/golden/make_golden.py   (writes the JSON files beside it)
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def hexs(v):
    return [float(x).hex() for x in v]


# --- the reference's arithmetic in plain Python --------------------------
class Sys:
    def __init__(self, box, x, y, z, vx=None, vy=None, vz=None, api=None, rc=2.5,
                 rskin=2.8, atskin=1.5, dt=0.005, nbtim=10, sig=(1.0, 1.0), eps=(1.0, 1.0),
                 mas=(1.0, 1.0)):
        n = len(x)
        self.n, self.L = n, box
        self.x, self.y, self.z = list(x), list(y), list(z)
        self.vx = list(vx) if vx else [0.0] * n
        self.vy = list(vy) if vy else [0.0] * n
        self.vz = list(vz) if vz else [0.0] * n
        self.ax, self.ay, self.az = [0.0] * n, [0.0] * n, [0.0] * n
        self.api = list(api) if api else [1] * n
        self.rc, self.atrskin, self.atskin, self.dt, self.nbtim = rc, rskin, atskin, dt, nbtim
        self.sig, self.eps, self.mas = sig, eps, mas
        # read-3d.f:263-276
        self.dmmh = [(rskin - rc) / float(nbtim)] * 256
        self.dmmsu = 256.0 * (rskin - rc) / float(nbtim)
        self.dmms, self.dmmst, self.dmmi, self.dmmax = 0.0, 0, 0, 0.0
        self.nlist, self.nidx = [], []
        self.epot = self.ekin = 0.0
        self.nrebuild = 0

    # neighbor-pbc-mav.f:13-109 (all pairs)
    def neighbor(self, step):
        L, ib = self.L, 1.0 / self.L
        if self.dmms > (self.atrskin - self.rc):
            raise RuntimeError("skin radius exceeded")  # :48-51
        if step != 0 and step > 0:
            self.atrskin = self.rc + (self.atrskin - self.rc) * float(self.nbtim) / float(self.dmmst)
            self.atrskin = min(L / 2.0, self.atrskin)
        rs2 = self.atrskin * self.atrskin
        for i in range(self.n):
            self.x[i] = math.fmod(math.fmod(self.x[i], L) + L, L)
            self.y[i] = math.fmod(math.fmod(self.y[i], L) + L, L)
            self.z[i] = math.fmod(math.fmod(self.z[i], L) + L, L)
        lst, idx = [], []
        for i in range(self.n):
            idx.append(len(lst) + 1)
            lst.append(-(i + 1))
            for j in range(i + 1, self.n):
                dx = self.x[i] - self.x[j]
                dy = self.y[i] - self.y[j]
                dz = self.z[i] - self.z[j]
                dx = dx + L - L * float(int(1.5 + dx * ib))
                dy = dy + L - L * float(int(1.5 + dy * ib))
                dz = dz + L - L * float(int(1.5 + dz * ib))
                if dx * dx + dy * dy + dz * dz <= rs2:
                    lst.append(j + 1)
        self.nlist, self.nidx = lst, idx
        self.dmmax = max(self.dmms, self.dmmax)
        self.dmms, self.dmmst = 0.0, 0
        self.nrebuild += 1

    def _mi(self, d, bf1, bf2):
        return d + self.L * (bf1 - float(int(bf2 + d * (1.0 / self.L))))

    # for-a-lj-n-pbc-m.f:18-154
    def accatom(self):
        s1, s2 = self.sig
        c111 = s1 * s1 * s1 * s1 * s1 * s1
        c112 = c111 * c111
        c113 = 0.5 * c111
        c221 = s2 * s2 * s2 * s2 * s2 * s2
        c222 = c221 * c221
        c223 = 0.5 * c221
        c121 = 0.5 * (s1 + s2)
        c121 = c121 * c121 * c121 * c121 * c121 * c121
        c122 = c121 * c121
        c123 = 0.5 * c121
        e11, e22 = self.eps
        e12 = math.sqrt(e11 * e22)
        coef = {2: (e11, c111, c112, c113), 3: (e12, c121, c122, c123), 4: (e22, c221, c222, c223)}
        bf1 = 2.0 + float(int(self.atrskin / s1))
        bf2 = bf1 + 0.5
        atr2 = self.rc * self.rc
        fs = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        esum = 0.0
        k = 0
        lst = self.nlist
        while True:
            i = -lst[k] - 1
            if i == self.n - 1:
                break
            k += 1
            while k < len(lst) and lst[k] > 0:
                j = lst[k] - 1
                k += 1
                dx = self._mi(self.x[i] - self.x[j], bf1, bf2)
                dy = self._mi(self.y[i] - self.y[j], bf1, bf2)
                dz = self._mi(self.z[i] - self.z[j], bf1, bf2)
                r2 = dx * dx + dy * dy + dz * dz
                if r2 <= atr2:
                    r2 = 1.0 / r2
                    r6 = r2 * r2 * r2
                    e, c1, c2, c3 = coef[self.api[i] + self.api[j]]
                    fij = e * 48.0 * r2 * r6 * (c2 * r6 - c3)
                    esum = esum + e * 4.0 * r6 * (c2 * r6 - c1)
                    fs[i][0] = fs[i][0] + fij * dx
                    fs[j][0] = fs[j][0] - fij * dx
                    fs[i][1] = fs[i][1] + fij * dy
                    fs[j][1] = fs[j][1] - fij * dy
                    fs[i][2] = fs[i][2] + fij * dz
                    fs[j][2] = fs[j][2] - fij * dz
        self.epot = esum
        for i in range(self.n):
            iatm = 1.0 / self.mas[self.api[i] - 1]
            self.ax[i] = self.ax[i] + fs[i][0] * iatm
            self.ay[i] = self.ay[i] + fs[i][1] * iatm
            self.az[i] = self.az[i] + fs[i][2] * iatm

    # int-verlet-mav.f:18-95
    def integrator(self, step):
        dt = self.dt
        dmmr = 0.0
        for i in range(self.n):
            dx = (self.vx[i] + 0.5 * self.ax[i] * dt) * dt
            dy = (self.vy[i] + 0.5 * self.ay[i] * dt) * dt
            dz = (self.vz[i] + 0.5 * self.az[i] * dt) * dt
            self.x[i] = self.x[i] + dx
            self.y[i] = self.y[i] + dy
            self.z[i] = self.z[i] + dz
            self.vx[i] = self.vx[i] + 0.5 * self.ax[i] * dt
            self.vy[i] = self.vy[i] + 0.5 * self.ay[i] * dt
            self.vz[i] = self.vz[i] + 0.5 * self.az[i] * dt
            dmmr = max(dmmr, dx * dx + dy * dy + dz * dz)
        dmmr = 2.2 * math.sqrt(dmmr)
        self.dmms = self.dmms + dmmr
        self.dmmsu = self.dmmsu + dmmr - self.dmmh[self.dmmi]
        self.dmmh[self.dmmi] = dmmr
        self.dmmi = (self.dmmi + 1) & 255
        self.dmmst += 1
        if self.dmms > (self.atrskin - self.rc - 2.0 * self.dmms / float(self.dmmst)):
            self.neighbor(step)
        self.ax, self.ay, self.az = [0.0] * self.n, [0.0] * self.n, [0.0] * self.n
        self.accatom()
        self.ekin = 0.0
        for i in range(self.n):
            self.vx[i] = self.vx[i] + 0.5 * self.ax[i] * dt
            self.vy[i] = self.vy[i] + 0.5 * self.ay[i] * dt
            self.vz[i] = self.vz[i] + 0.5 * self.az[i] * dt
            m = self.mas[self.api[i] - 1]
            self.ekin = self.ekin + 0.5 * m * (self.vx[i] * self.vx[i] + self.vy[i] * self.vy[i]
                                               + self.vz[i] * self.vz[i])

    def _bonds(self, species_filter):
        """stoddard-pbc-n-m.f:70-104 (species_filter) / -fre.f:84-117."""
        bf1 = float(int(self.atrskin / self.sig[0])) + 2.0
        bf2 = bf1 + 0.5
        rc2 = self.atskin * self.atskin
        adj = [[] for _ in range(self.n)]
        for i in range(self.n - 1):
            if species_filter and self.api[i] != 1:
                continue
            k = self.nidx[i]  # 1-based header position; entries follow
            while k < len(self.nlist) and self.nlist[k] > 0:
                j = self.nlist[k] - 1
                k += 1
                if species_filter and self.api[j] != 1:
                    break
                dx = self._mi(self.x[i] - self.x[j], bf1, bf2)
                dy = self._mi(self.y[i] - self.y[j], bf1, bf2)
                dz = self._mi(self.z[i] - self.z[j], bf1, bf2)
                if dx * dx + dy * dy + dz * dz <= rc2:
                    adj[i].append(j)
                    adj[j].append(i)
        return adj

    def stillinger(self):
        """Connected components; label = smallest atom number; sizes; csi(1:)."""
        adj = self._bonds(True)
        lab = [0] * self.n
        for k in range(self.n):
            if lab[k]:
                continue
            stack = [k]
            lab[k] = k + 1
            while stack:
                a = stack.pop()
                for b in adj[a]:
                    if not lab[b]:
                        lab[b] = k + 1
                        stack.append(b)
        cs = [0] * self.n
        for i in range(self.n):
            cs[lab[i] - 1] += 1
        csi = [0] * (self.n + 1)
        for c in cs:
            if c:
                csi[c] += 1
        csi[0] = self.n - sum(1 for c in cs if c)  # first call: the never-reset csi(0)
        return lab, cs, csi

    def frenkel(self, atnenum):
        """Liquid atoms and their components (stoddard-pbc-n-m-fre.f:143-225):
        label = 1-based rank of the component's smallest liquid atom."""
        adj = self._bonds(False)
        liq = [self.api[k] == 1 and len(adj[k]) >= atnenum and
               sum(1 for m in adj[k] if self.api[m] == 1) >= atnenum for k in range(self.n)]
        rank = {}
        for k in range(self.n):
            if liq[k]:
                rank[k] = len(rank) + 1
        lab = [0] * self.n
        for k in range(self.n):
            if not liq[k] or lab[k]:
                continue
            stack = [k]
            lab[k] = rank[k]
            while stack:
                a = stack.pop()
                for b in adj[a]:
                    if liq[b] and not lab[b]:
                        lab[b] = rank[k]
                        stack.append(b)
        return liq, lab


def fixture(name, s, steps=0, clusters=True, frenkel=None, extra=None):
    d = {"name": name, "n": s.n, "box": s.L.hex(), "api": s.api, "rskin": s.atrskin.hex(),
         "sig": hexs(s.sig), "eps": hexs(s.eps), "mas": hexs(s.mas),
         "x0": hexs(s.x), "y0": hexs(s.y), "z0": hexs(s.z),
         "vx0": hexs(s.vx), "vy0": hexs(s.vy), "vz0": hexs(s.vz)}
    s.neighbor(0)
    s.accatom()
    d.update({"atnlist": s.nlist, "atnidx": s.nidx, "epot": s.epot.hex(),
              "ax": hexs(s.ax), "ay": hexs(s.ay), "az": hexs(s.az),
              "xw": hexs(s.x), "yw": hexs(s.y), "zw": hexs(s.z)})
    if clusters:
        lab, cs, csi = s.stillinger()
        d.update({"cl": lab, "cs": cs, "csi": csi})
    if frenkel:
        liq, labf = s.frenkel(frenkel)
        d.update({"atnenum": frenkel, "liquid": [int(v) for v in liq], "clf": labf})
    if steps:
        for i in range(1, steps + 1):
            s.integrator(i)
        d.update({"steps": steps, "x": hexs(s.x), "y": hexs(s.y), "z": hexs(s.z),
                  "vx": hexs(s.vx), "vy": hexs(s.vy), "vz": hexs(s.vz),
                  "ekin": s.ekin.hex(), "epot_end": s.epot.hex(), "nrebuild": s.nrebuild,
                  "atrskin": s.atrskin.hex()})
    if extra:
        d.update(extra)
    return d


def lcg(seed):
    """Small deterministic generator (not the engine's) for the fixtures."""
    state = seed
    while True:
        state = (6364136223846793005 * state + 1442695040888963407) % (1 << 64)
        yield (state >> 11) / float(1 << 53)


def main():
    out = []
    # 1. LJ pair known answers: minimum, zero crossing, cut-off and list edges.
    # Box and offsets are dyadic, so the reference's minimum-image arithmetic
    # reproduces r exactly and r^2 == rc^2 / rs^2 really is the edge case.
    r_min = 2.0 ** (1.0 / 6.0)
    tiny = 2.0 ** -30
    for tag, r in [("min", r_min), ("sigma", 1.0), ("rc", 2.5), ("beyond_rc", 2.5 + tiny),
                   ("rs", 2.75), ("beyond_rs", 2.75 + tiny)]:
        s = Sys(16.0, [4.0, 4.0 + r], [4.0, 4.0], [5.0, 5.0], rskin=2.75)
        out.append(fixture(f"pair_{tag}", s, clusters=False, extra={"r": r.hex()}))
    # 2. four atoms on a line (the layout of init-2atom.f:41-69, reduced units)
    c = 10.0
    s = Sys(20.0, [c + 3.0, c - 3.0, c - 0.6, c + 0.6], [c] * 4, [c] * 4,
            vx=[0.3, -0.3, 0.0, 0.0])
    out.append(fixture("line4", s, steps=40))
    # 3. a tetrahedron around the box corner (its atoms sit in four different
    # corners of the box) plus atoms across faces and edges, all given
    # outside [0, L) so the wrap and every minimum image are exercised
    L = 9.0
    h = 0.55
    pts = [(-h, -h, -h), (L + h, L + h, -h), (L + h, -h, L + h), (-h, L + h, L + h),
           (4.5, -0.6, 4.5), (4.5, L + 0.7, 4.5), (-0.7, 4.5, L + 0.6)]
    s = Sys(L, [p[0] for p in pts], [p[1] for p in pts], [p[2] for p in pts])
    out.append(fixture("corners8", s, steps=20))
    # 4. a chain of bonded atoms through the periodic boundary + monomers
    L = 16.0
    xs = [L - 2.8, L - 1.4, 0.0 + 1e-3, 1.4, 2.8, 8.0, 8.0, 12.0]
    ys = [4.0, 4.0, 4.0, 4.0, 4.0, 8.0, 9.45, 12.0]
    zs = [4.0, 4.0, 4.0, 4.0, 4.0, 8.0, 8.0, 2.0]
    order = [6, 2, 7, 0, 4, 1, 5, 3]  # scramble so labels are not 1..n
    s = Sys(L, [xs[k] for k in order], [ys[k] for k in order], [zs[k] for k in order])
    out.append(fixture("chain_pbc", s))
    # 5. species 2 ends a Stillinger row (stoddard-pbc-n-m.f:85)
    s = Sys(16.0, [5.0, 6.2, 5.6, 7.4], [5.0, 5.0, 5.9, 5.0], [5.0] * 4, api=[1, 2, 1, 1],
            sig=(1.0, 0.9), eps=(1.0, 0.5), mas=(1.0, 0.2))
    out.append(fixture("species2_row_end", s))
    # 6. a 13-atom icosahedral blob + vapour: ten Wolde-Frenkel liquid atoms
    L = 18.0
    phi = (1 + 5 ** 0.5) / 2
    ico = []
    for a in (-1, 1):
        for b in (-1, 1):
            ico += [(0, a, b * phi), (a, b * phi, 0), (b * phi, 0, a)]
    sc = 1.1 / math.sqrt(1 + phi * phi)
    blob = [(6.0, 6.0, 6.0)] + [(6.0 + sc * p[0], 6.0 + sc * p[1], 6.0 + sc * p[2]) for p in ico]
    vap = [(14.0, 3.0, 9.0), (2.0, 14.5, 15.0), (10.0, 12.0, 1.0)]
    allp = blob + vap
    s = Sys(L, [p[0] for p in allp], [p[1] for p in allp], [p[2] for p in allp])
    out.append(fixture("frenkel_blob", s, frenkel=5))
    # 7. 48 random atoms (all pairs >= 0.9 apart), 30 VV steps
    g = lcg(12345)
    L = 5.5
    pts = []
    while len(pts) < 48:
        p = (next(g) * L, next(g) * L, next(g) * L)
        ok = True
        for q in pts:
            d = [p[k] - q[k] for k in range(3)]
            d = [dd - L * round(dd / L) for dd in d]
            if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 0.81:
                ok = False
                break
        if ok:
            pts.append(p)
    vs = [((next(g) - 0.5), (next(g) - 0.5), (next(g) - 0.5)) for _ in pts]
    s = Sys(L, [p[0] for p in pts], [p[1] for p in pts], [p[2] for p in pts],
            vx=[v[0] for v in vs], vy=[v[1] for v in vs], vz=[v[2] for v in vs])
    out.append(fixture("random48", s, steps=30))
    for d in out:
        with open(os.path.join(HERE, d["name"] + ".json"), "w") as f:
            json.dump(d, f, indent=0)
    print(f"wrote {len(out)} fixtures")


if __name__ == "__main__":
    main()
