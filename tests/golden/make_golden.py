"""Generate the golden fixtures in tests/golden/ from a second, independent
pure-Python restatement of the reference's serial Fortran loops, written
directly from the Fortran with 1-based indices (small cases only):

  parcel_mixing.F90:68-431 + construct_grids :440-624  (mix_case.npz)
  parcels/haloswap.F90:109-289                         (haloswap_case.npz)
  parcel_splitting.F90:47-168                          (split_case.npz)
  parcel_interpolation.F90:186-481 (par2grid)          (par2grid_case.npz)

The C++ oracle and the GPU library are both checked against these vectors.
Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
F32 = lambda a, b: float(np.float32(np.float32(a) / np.float32(b)))  # REAL(4) a/b widened


class Geo:
    """setup_grid.F90:45-104 and parcel_interpolation.F90:76-136, one rank."""

    def __init__(self, Nx, Ny, Nz, Lx, Ly, Lz):
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.nzp = Nz + 1
        self.dx, self.dy, self.dz = Lx / Nx, Ly / Ny, Lz / (self.nzp - 1)
        self.nx, self.ny, self.nz = Nx + 4, Ny + 4, self.nzp
        self.xmin = (-1 - 1) * self.dx + 0.0
        self.ymin = (-1 - 1) * self.dy + 0.0
        self.zmin = 0 * self.dz + 0.0
        self.zmax = (self.nzp - 1) * self.dz
        self.xc = [None] + [self.xmin + (n - 1) * self.dx + 0.0 for n in range(1, self.nx + 1)]
        self.yc = [None] + [self.ymin + (n - 1) * self.dy + 0.0 for n in range(1, self.ny + 1)]
        self.zc = [None] + [self.zmin + (n - 1) * self.dz + 0.0 for n in range(1, self.nz + 1)]
        self.top = (Lx - self.dx, Ly - self.dy)
        self.vmin = self.dx * self.dy * self.dz / 6. / 6. / 6.

    def grid(self):
        return np.zeros((self.nz + 1, self.ny + 1, self.nx + 1))  # 1-based (k, j, i)

    def bin(self, x, y, z):
        i = math.floor((x - self.xmin) / self.dx) + 1
        j = math.floor((y - self.ymin) / self.dy) + 1
        k = math.floor((z - self.zmin) / self.dz) + 1
        assert 1 <= i < self.nx and 1 <= j < self.ny and 1 <= k < self.nz
        delx = ((x - self.xmin) - (i - 1) * self.dx) / self.dx
        dely = ((y - self.ymin) - (j - 1) * self.dy) / self.dy
        delz = ((z - self.zmin) - (k - 1) * self.dz) / self.dz
        return i, j, k, delx, dely, delz

    def halo_sum(self, a):  # par2grid_haloswap, MPIC_Haloswap.F90:188-290
        xi, xf, yi, yf = 3, self.Nx + 2, 3, self.Ny + 2
        right = a[1:, yi:yf + 1, xf + 1].copy()
        up = a[1:, yf + 1, xi:xf + 1].copy()
        corner = a[1:, yf + 1, xf + 1].copy()
        a[1:, yi:yf + 1, xi] += right
        a[1:, yi, xi:xf + 1] += up
        a[1:, yi, xi] += corner

    def halo_copy(self, a):  # grid2par_haloswap, :95-184
        xi, xf, yi, yf = 3, self.Nx + 2, 3, self.Ny + 2
        left = a[1:, yi:yf + 1, xi].copy()
        down = a[1:, yi, xi:xf + 1].copy()
        corner = a[1:, yi, xi].copy()
        a[1:, yi:yf + 1, xf + 1] = left
        a[1:, yf + 1, xi:xf + 1] = down
        a[1:, yf + 1, xf + 1] = corner

    def interior(self, a):
        return a[1:self.nzp + 1, 3:self.Ny + 3, 3:self.Nx + 3].copy()


def weights(delx, dely, delz, v):
    return [(1 - delz) * (1 - dely) * (1 - delx) * v, (1 - delz) * (1 - dely) * (delx) * v,
            (1 - delz) * (dely) * (1 - delx) * v, (1 - delz) * (dely) * (delx) * v,
            (delz) * (1 - dely) * (1 - delx) * v, (delz) * (1 - dely) * (delx) * v,
            (delz) * (dely) * (1 - delx) * v, (delz) * (dely) * (delx) * v]


CORNERS = [(0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)]  # (dk,dj,di)


def par2grid(G, P, var):
    W, D = G.grid(), G.grid()
    for n in range(len(P["x"])):
        i, j, k, dx, dy, dz = G.bin(P["x"][n], P["y"][n], P["z"][n])
        w = weights(dx, dy, dz, P["vol"][n])
        for c, (a, b, e) in enumerate(CORNERS):
            D[k + a, j + b, i + e] = D[k + a, j + b, i + e] + w[c] * var[n]
            W[k + a, j + b, i + e] = W[k + a, j + b, i + e] + w[c]
    G.halo_sum(W)
    G.halo_sum(D)
    W[W == 0.] = 1.
    return G.interior(D / W)


def mixing(G, P, n_slots):
    """parcel_mixing.F90:68-431 for one rank, slots 1-based, arrays of capacity n_slots."""
    norig = P["n"]
    keep = [None] + [0] * norig
    npc = np.zeros((G.nz, G.ny, G.nx), int)  # npercell(nz-1, ny-1, nx-1), 1-based
    names = ["vol", "b", "h", "p", "q", "r"]
    K = {q: G.grid() for q in names}
    R = {q: G.grid() for q in names}
    cache = [None]
    nremove = 0
    for n in range(1, norig + 1):  # construct_grids :469-621
        i, j, k, dx, dy, dz = G.bin(P["x"][n - 1], P["y"][n - 1], P["z"][n - 1])
        cache.append((i, j, k, dx, dy, dz))
        v = P["vol"][n - 1]
        w = weights(dx, dy, dz, v)
        if P["vol"][n - 1] < G.vmin:
            keep[n] = 0
            nremove += 1
            tgt = R
        else:
            keep[n] = 1
            npc[k, j, i] += 1
            tgt = K
        for q in names:
            f = 1.0 if q == "vol" else P[q][n - 1]
            for c, (a, b, e) in enumerate(CORNERS):
                g = tgt[q]
                g[k + a, j + b, i + e] = g[k + a, j + b, i + e] + (w[c] if q == "vol" else w[c] * f)
    for q in names:
        G.halo_sum(K[q])
        G.halo_copy(K[q])
        K[q][1, :, :] = K[q][1, :, :] * 2.
        K[q][G.nz, :, :] = K[q][G.nz, :, :] * 2
    nadd = 0
    n = 1
    numloc = norig
    new_slots = []
    for i in range(3, G.nx - 2 + 1):  # :160-212
        for j in range(3, G.ny - 2 + 1):
            for k in range(1, G.nz - 1 + 1):
                if npc[k, j, i] < 3:
                    nadd += 1
                    if n <= numloc:
                        while keep[n] != 0:
                            n = n + 1
                            if n > numloc:
                                break
                    box = lambda g: sum(g[kk, jj, ii] for ii in (i, i + 1) for jj in (j, j + 1) for kk in (k, k + 1))
                    v = box(K["vol"])
                    portion = 2 * G.vmin / v
                    s = n - 1
                    P["x"][s] = 0.5 * (G.xc[i] + G.xc[i + 1])
                    P["y"][s] = 0.5 * (G.yc[j] + G.yc[j + 1])
                    P["z"][s] = 0.5 * (G.zc[k] + G.zc[k + 1])
                    P["vol"][s] = 2 * G.vmin
                    P["stretch"][s] = 0
                    for q in ["b", "h", "p", "q", "r"]:
                        P[q][s] = box(K[q]) / v
                    if n < numloc:
                        keep[n] = 2
                    new_slots.append(s)
                    n = n + 1
                    assert n <= n_slots
                    for q in names:
                        for ii in (i, i + 1):
                            for jj in (j, j + 1):
                                for kk in (k, k + 1):
                                    R[q][kk, jj, ii] = R[q][kk, jj, ii] - portion * K[q][kk, jj, ii]
    count = max(n - 1, numloc)
    for q in names:
        G.halo_sum(R[q])
        G.halo_copy(R[q])
        R[q][1, :, :] = R[q][1, :, :] * 2
        R[q][G.nz, :, :] = R[q][G.nz, :, :] * 2
    for m in range(1, norig + 1):  # :247-340
        if keep[m] != 1:
            continue
        i, j, k, dx, dy, dz = cache[m]
        v = P["vol"][m - 1]
        w = weights(dx, dy, dz, v)
        V = K["vol"]
        nv = P["vol"][m - 1]
        for c, (a, b, e) in enumerate(CORNERS):
            nv = nv + w[c] * R["vol"][k + a, j + b, i + e] / V[k + a, j + b, i + e]
        P["vol"][m - 1] = nv
        for q in ["b", "h", "p", "q", "r"]:
            s = P[q][m - 1] * v
            for c, (a, b, e) in enumerate(CORNERS):
                s = s + w[c] / V[k + a, j + b, i + e] * R[q][k + a, j + b, i + e]
            P[q][m - 1] = s / nv
    if count == norig:  # :347-389
        last = norig
        for m in range(1, norig + 1):
            if keep[m] == 0:
                while keep[last] != 1:
                    last -= 1
                    assert last >= 1
                for q in ["x", "y", "z", "p", "q", "r", "b", "h", "vol", "tag", "stretch"]:
                    P[q][m - 1] = P[q][last - 1]
                last -= 1
                count -= 1
    P["n"] = count
    return dict(nremove=nremove, nadd=nadd, keep=np.array(keep[1:]), npc=npc, new_slots=np.array(new_slots))


def haloswap(G, P):
    """parcels/haloswap.F90:109-289, one rank."""
    n0 = P["n"]
    for i in range(n0):  # reflect :440-456
        z = P["z"][i]
        if z < G.zmin:
            P["z"][i] = G.zmin + (G.zmin - z)
        elif z > G.zmax:
            P["z"][i] = G.zmax - (z - G.zmax)
    ymax, ymin = G.yc[G.ny - 2 + 1], G.yc[2 + 1]
    xmax, xmin = G.xc[G.nx - 2 + 1], G.xc[2 + 1]
    index = [0] * n0
    for d in range(1, 9):  # count_parcels_to_send :296-437
        for i in range(n0):
            x, y = P["x"][i], P["y"][i]
            hit = {1: y >= ymax and xmin <= x < xmax, 5: y < ymin and xmin <= x < xmax,
                   3: x >= xmax and ymin <= y < ymax, 7: x < xmin and ymin <= y < ymax,
                   2: x >= xmax and y >= ymax, 8: x < xmin and y >= ymax,
                   4: x >= xmax and y < ymin, 6: x < xmin and y < ymin}[d]
            if hit:
                index[i] = d
    props = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt", "h", "b", "vol",
             "stretch", "tag", "xo", "yo", "zo", "xf", "yf", "zf", "po", "qo", "ro", "pf", "qf", "rf"]
    bottom = (0.0, 0.0)
    msgs = []
    for d in range(1, 9):  # populate_send_buffer :489-607
        xs = ys = 0.0
        if d in (3, 2, 4):
            xs = bottom[0] - G.top[0] - G.dx
        elif d in (7, 8, 6):
            xs = G.top[0] - bottom[0] + G.dx
        if d in (1, 2, 8):
            ys = bottom[1] - G.top[1] - G.dy
        elif d in (5, 6, 4):
            ys = G.top[1] - bottom[1] + G.dy
        for i in range(n0):
            if index[i] == d:
                rec = {}
                for q in props:
                    v = P[q][i]
                    if q in ("x", "xo", "xf"):
                        v = v + xs
                    if q in ("y", "yo", "yf"):
                        v = v + ys
                    rec[q] = v
                msgs.append(rec)
    last = 1  # unpack_parcels :678-771
    idx1 = [None] + index
    for rec in msgs:
        i = last
        while not (i > n0 or idx1[i] != 0):
            i += 1
        idx1[i] = 0
        for q in props:
            P[q][i - 1] = rec[q]
        last = i + 1
    return np.array(index)


def splitting(P, dt):
    """parcel_splitting.F90:64-137."""
    third = F32(1., 3.)
    pi = 4. * math.atan(1.0)
    n = P["n"]
    for i in range(P["n"]):
        ds = P["p"][i] * P["dpdt"][i] + P["q"][i] * P["dqdt"][i] + P["r"][i] * P["drdt"][i]
        ds = abs(ds) ** third
        P["stretch"][i] = P["stretch"][i] + ds * dt
        if P["stretch"][i] > 4.:
            r = P["vol"][i] / 4. / pi
            r = r ** third
            absw = math.sqrt(P["p"][i] ** 2 + P["q"][i] ** 2 + P["r"][i] ** 2)
            c = n
            n += 1
            for q in ["p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt", "h", "b", "tag"]:
                P[q][c] = P[q][i]
            P["x"][c] = P["x"][i] + r * P["p"][i] / absw
            P["y"][c] = P["y"][i] + r * P["q"][i] / absw
            P["z"][c] = P["z"][i] + r * P["r"][i] / absw
            P["vol"][c] = P["vol"][i] / 2
            P["stretch"][c] = 0.
            P["x"][i] = P["x"][i] - r * P["p"][i] / absw
            P["y"][i] = P["y"][i] - r * P["q"][i] / absw
            P["z"][i] = P["z"][i] - r * P["r"][i] / absw
            P["vol"][i] = P["vol"][i] / 2
            P["stretch"][i] = 0.
    P["n"] = n


ALL = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt", "h", "b", "vol",
       "stretch", "tag", "xo", "yo", "zo", "xf", "yf", "zf", "po", "qo", "ro", "pf", "qf", "rf"]


def random_parcels(G, rng, n, cap, Lx, Ly, Lz):
    P = {q: np.zeros(cap) for q in ALL}
    P["x"][:n] = rng.uniform(0, Lx, n)
    P["y"][:n] = rng.uniform(0, Ly, n)
    P["z"][:n] = rng.uniform(0.01 * Lz, 0.99 * Lz, n)
    for q in ["p", "q", "r", "b", "h", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt"]:
        P[q][:n] = rng.standard_normal(n)
    P["vol"][:n] = G.dx * G.dy * G.dz / 8 * rng.uniform(0.5, 1.5, n)
    P["tag"][:n] = np.arange(n)
    P["n"] = n
    return P


def main():
    rng = np.random.default_rng(2024)
    Nx, Ny, Nz, Lx, Ly, Lz = 6, 4, 5, 2 * math.pi, 2 * math.pi, math.pi
    # ---- mixing: 5 parcels/cell on average, clustered so that some cells are
    # under-populated, ~15% of parcels below vmin
    G = Geo(Nx, Ny, Nz, Lx, Ly, Lz)
    n = 5 * Nx * Ny * Nz
    cap = 3 * n
    P = random_parcels(G, rng, n, cap, Lx, Ly, Lz)
    P["x"][:n] = np.where(rng.uniform(size=n) < 0.5, rng.uniform(0, 0.6 * Lx, n), P["x"][:n])
    small = rng.uniform(size=n) < 0.15
    P["vol"][:n][small] = G.vmin * rng.uniform(0.2, 0.95, small.sum())
    inp = {q: P[q].copy() for q in ALL}
    out = mixing(G, P, cap)
    np.savez_compressed(os.path.join(HERE, "mix_case.npz"), geom=np.array([Nx, Ny, Nz, Lx, Ly, Lz]), n_in=n, cap=cap,
             n_out=P["n"], nremove=out["nremove"], nadd=out["nadd"], keep=out["keep"],
             new_slots=out["new_slots"], **{"in_" + q: inp[q] for q in ALL}, **{"out_" + q: P[q] for q in ALL})
    # ---- mixing where new parcels exactly fill the removed slots including the
    # last slot (the strict `n < numparcels_local` case) is exercised by a
    # second, hand-shaped case: the last slot is removed and the number of
    # under-populated cells equals the number of removed parcels
    G2 = Geo(4, 4, 3, Lx, Ly, Lz)
    nc = 4 * 4 * 3
    per = 4
    n2 = nc * per
    P2 = {q: np.zeros(3 * n2) for q in ALL}
    t = 0
    for i in range(4):
        for j in range(4):
            for k in range(3):
                for s in range(per):
                    P2["x"][t] = (i + rng.uniform(0.05, 0.95)) * G2.dx
                    P2["y"][t] = (j + rng.uniform(0.05, 0.95)) * G2.dy
                    P2["z"][t] = (k + rng.uniform(0.05, 0.95)) * G2.dz
                    t += 1
    for q in ["p", "q", "r", "b", "h"]:
        P2[q][:n2] = rng.standard_normal(n2)
    P2["vol"][:n2] = G2.dx * G2.dy * G2.dz / per
    P2["tag"][:n2] = np.arange(n2)
    # cells (0,0,0) (slots 0..3) and (0,0,1) (slots 4..7) each lose two
    # parcels to the last cell -> two under-populated cells -> two new parcels;
    # exactly two parcels are removed, in the last two slots, so the second new
    # parcel lands in the last slot and keeps keep = 0 (`n < numparcels_local`
    # is strict), after which the backfill overwrites it
    for s in [0, 1, 4, 5]:
        P2["x"][s] = P2["x"][n2 - 1]
        P2["y"][s] = P2["y"][n2 - 1]
        P2["z"][s] = P2["z"][n2 - 1]
    P2["vol"][[n2 - 2, n2 - 1]] = G2.vmin * 0.5
    P2["n"] = n2
    inp2 = {q: P2[q].copy() for q in ALL}
    out2 = mixing(G2, P2, 3 * n2)
    np.savez_compressed(os.path.join(HERE, "mix_case_last_slot.npz"), geom=np.array([4, 4, 3, Lx, Ly, Lz]), n_in=n2,
             cap=3 * n2, n_out=P2["n"], nremove=out2["nremove"], nadd=out2["nadd"], keep=out2["keep"],
             new_slots=out2["new_slots"], **{"in_" + q: inp2[q] for q in ALL},
             **{"out_" + q: P2[q] for q in ALL})
    # ---- haloswap: parcels pushed across every face and corner
    G = Geo(Nx, Ny, Nz, Lx, Ly, Lz)
    n = 400
    P = random_parcels(G, rng, n, 2 * n, Lx, Ly, Lz)
    for q in ["xo", "yo", "zo", "xf", "yf", "zf", "po", "qo", "ro", "pf", "qf", "rf"]:
        P[q][:n] = rng.standard_normal(n)
    sel = rng.uniform(size=n) < 0.7
    P["x"][:n][sel] = rng.uniform(-0.15 * Lx, 1.15 * Lx, sel.sum())
    P["y"][:n][sel] = rng.uniform(-0.15 * Ly, 1.15 * Ly, sel.sum())
    sel = rng.uniform(size=n) < 0.1
    P["z"][:n][sel] = np.where(rng.uniform(size=sel.sum()) < 0.5, -rng.uniform(0, 0.1, sel.sum()),
                               Lz + rng.uniform(0, 0.1, sel.sum()))
    inp = {q: P[q].copy() for q in ALL}
    index = haloswap(G, P)
    np.savez_compressed(os.path.join(HERE, "haloswap_case.npz"), geom=np.array([Nx, Ny, Nz, Lx, Ly, Lz]), n_in=n,
             cap=2 * n, index=index, **{"in_" + q: inp[q] for q in ALL}, **{"out_" + q: P[q] for q in ALL})
    # ---- splitting
    n = 300
    P = random_parcels(G, rng, n, 3 * n, Lx, Ly, Lz)
    P["stretch"][:n] = rng.uniform(3.0, 4.2, n)
    dt = 0.05
    inp = {q: P[q].copy() for q in ALL}
    splitting(P, dt)
    haloswap(G, P)  # parcel_splitting.F90:158
    np.savez_compressed(os.path.join(HERE, "split_case.npz"), geom=np.array([Nx, Ny, Nz, Lx, Ly, Lz]), n_in=n,
             cap=3 * n, dt=dt, n_out=P["n"], **{"in_" + q: inp[q] for q in ALL},
             **{"out_" + q: P[q] for q in ALL})
    # ---- par2grid
    n = 400
    P = random_parcels(G, rng, n, n, Lx, Ly, Lz)
    g = par2grid(G, P, P["b"][:n])
    np.savez_compressed(os.path.join(HERE, "par2grid_case.npz"), geom=np.array([Nx, Ny, Nz, Lx, Ly, Lz]), n_in=n,
             **{"in_" + q: P[q] for q in ALL}, grid=g)
    print("fixtures written")


if __name__ == "__main__":
    main()
