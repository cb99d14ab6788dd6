"""FP64 oracle of the incompressible Navier-Stokes path (test infrastructure only).

A numpy restatement, vectorised over cell-face entries, of what
graphite_b200's FvmNSI* / gbNSIRun compute: artificial compressibility
(dp/dt + beta^2 div u = 0, du/dt + div(u u + p I) - nu lap u = 0) with
least-squares gradients (the reference's LSQ, src/fvmops.cu:51-111), the
reference's limiter (src/fvmops.cu:129-169) when asked for, second-order
reconstruction,
a Rusanov flux with the wave speed |u.n| + sqrt((u.n)^2 + beta^2), the
viscous face gradient as the average of the cells' gradients
(fvmLaplacianC, include/fvmops.cuh:96-102) plus, optionally, the compact
correction along the centroid offset, and a local pseudo-time step.  The
reference defines no incompressible solver (src/models/nsi.cu calls
FvmNSI* functions that do not exist), so this oracle pins the scheme itself,
in float64, not a reference output.
"""
from __future__ import annotations

import numpy as np

from .pyoracle import OracleMesh


def limiter(u, g, umin, umax, d, k3):
    """Vectorised src/fvmops.cu:129-169 (a smooth switch between 1 and a
    Venkatakrishnan-type limiter of the face extrapolation g . d)."""
    delta = np.einsum("ij,ij->i", g, d)
    du, dd = umax - u, umin - u
    dmm2 = (du - dd) ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        y = dmm2 / k3 - 1.0
        sig = np.where(dmm2 <= k3, 1.0, np.where(dmm2 <= 2.0 * k3, 2 * y ** 3 - 3 * y ** 2 + 1.0, 0.0))
        yp = du / delta
        yn = dd / delta
        lp = np.where(yp < 2.0, yp - 0.25 * yp * yp, 1.0)
        ln = np.where(yn < 2.0, yn - 0.25 * yn * yn, 1.0)
    lim = np.where(delta > 1e-6, lp, np.where(delta < -1e-6, ln, 1.0)) * 0.8
    return sig + (1.0 - sig) * lim


class NSIOracle:
    def __init__(self, mesh: OracleMesh, viscosity=0.025, beta=2.0, corrected=True, density=1.0, limited=False):
        self.m = mesh
        self.limited = bool(limited)
        self.nu, self.beta2, self.corrected, self.density = float(viscosity), float(beta) ** 2, bool(corrected), density
        N, G = mesh.N, mesh.G
        self.N, self.G = N, G
        cfs, cf, cc = mesh.get("cell_faces_starts"), mesh.get("cell_faces"), mesh.get("cell_connects")
        self.area = mesh.get("face_areas")
        self.fn = mesh.get("face_normals").reshape(-1, 3)
        self.fc = mesh.get("face_centers").reshape(-1, 3)
        self.cc = mesh.get("cell_centers").reshape(-1, 3)
        self.vol = mesh.get("cell_volumes")
        self.gstart, self.gid = mesh.get("ghost_cell_starts"), mesh.get("ghost_cell_ids")
        counts = np.diff(cfs[: N + 1])
        self.ec = np.repeat(np.arange(N), counts)                 # entry -> cell
        self.ef = cf[cfs[0]:cfs[N]]                                # entry -> face
        self.ej = cc[cfs[0]:cfs[N]]                                # entry -> neighbour
        ci = self.cc[self.ec]
        self.d = self.cc[self.ej] - ci
        self.w2 = 1.0 / np.einsum("ij,ij->i", self.d, self.d)
        self.d0 = self.fc[self.ef] - ci
        self.d1 = self.fc[self.ef] - self.cc[self.ej]
        self.k3 = np.linalg.norm(self.d0, axis=1) ** 3
        s = np.einsum("ij,ij->i", self.fn[self.ef], self.d0)
        self.n = self.fn[self.ef] * np.where(s >= 0, 1.0, -1.0)[:, None]
        self.ds = self.area[self.ef] / self.vol[self.ec]
        # padded per-cell entry table (at most 6 faces per cell): cell sums as
        # row sums instead of scattered adds
        self.nf = counts
        self.pad = np.full((N, 6), -1, np.int64)
        slot = np.arange(len(self.ec)) - np.repeat(cfs[:N], counts)
        self.pad[self.ec, slot] = np.arange(len(self.ec))
        self.mask = self.pad >= 0
        self.padi = np.where(self.mask, self.pad, 0)
        A = self.cellsum(np.einsum("ij,ik->ijk", self.d, self.d) * self.w2[:, None, None])
        self.Ainv = np.linalg.inv(A)
        self.ghost_nb = self.ej >= N
        # ghost geometry: interior cell, face, normal out of the interior cell
        self.g_int = np.empty(G, np.int64)
        self.g_face = np.empty(G, np.int64)
        for t in range(G):
            c0 = self.gid[t]
            self.g_int[c0 - N] = cc[cfs[c0]]
            self.g_face[c0 - N] = cf[cfs[c0]]
        gi = self.g_int
        s = np.einsum("ij,ij->i", self.fn[self.g_face], self.fc[self.g_face] - self.cc[gi])
        self.g_n = self.fn[self.g_face] * np.where(s >= 0, 1.0, -1.0)[:, None]
        self.p = np.zeros(N + G)
        self.u = np.zeros((N + G, 3))

    def cellsum(self, x):
        """Per-cell sum of an entry array x[S, ...] (in entry order)."""
        y = x[self.padi]
        m = self.mask.reshape(self.mask.shape + (1,) * (x.ndim - 1))
        return np.where(m, y, 0.0).sum(axis=1)

    def cellmin(self, x, init):
        y = np.where(self.mask.reshape(self.mask.shape + (1,) * (x.ndim - 1)), x[self.padi], np.inf)
        return np.minimum(init, y.min(axis=1))

    def cellmax(self, x, init):
        y = np.where(self.mask.reshape(self.mask.shape + (1,) * (x.ndim - 1)), x[self.padi], -np.inf)
        return np.maximum(init, y.max(axis=1))

    def init(self, velocity, pressure):
        self.p[:] = pressure
        self.u[:] = np.asarray(velocity, np.float64)

    def apply_bcs(self, bcs):
        for b in bcs:
            r = self.m.region_id(b[1])
            ghosts = self.gid[self.gstart[r]:self.gstart[r + 1]]
            k = ghosts - self.N
            i, n = self.g_int[k], self.g_n[k]
            ui, pi = self.u[i], self.p[i]
            if b[0] == "slip":
                self.u[ghosts] = ui - n * (2 * np.einsum("ij,ij->i", n, ui))[:, None]
                self.p[ghosts] = pi
            elif b[0] == "wall":
                self.u[ghosts] = -ui
                self.p[ghosts] = pi
            else:
                vinf = np.asarray(b[2:5], np.float64)
                inflow = n @ vinf < 0
                self.u[ghosts] = np.where(inflow[:, None], vinf[None, :], ui)
                self.p[ghosts] = np.where(inflow, pi, float(b[5]))

    def gradients(self):
        """(gradients [N][4][3], limiters [N][4]) of p, u_x, u_y, u_z."""
        N = self.N
        v = np.column_stack([self.p, self.u])                     # (N+G, 4)
        vi, vj = v[self.ec], v[self.ej]
        sums = self.cellsum((vj - vi)[:, :, None] * self.d[:, None, :] * self.w2[:, None, None])
        g = np.einsum("nab,ncb->nca", self.Ainv, sums)
        vmin = self.cellmin(vj, v[:N])
        vmax = self.cellmax(vj, v[:N])
        lim = np.ones((N, 4))
        for c in range(4 if self.limited else 0):
            l = limiter(vi[:, c], g[self.ec, c], vmin[self.ec, c], vmax[self.ec, c], self.d0, self.k3)
            lim[:, c] = self.cellmin(l, np.full(N, 2.0))
        return g, lim

    def step(self, cfl):
        """One iteration after the boundary conditions; returns the residual
        sum of (R_p^2 + |R_u|^2) V."""
        N = self.N
        g, lim = self.gradients()
        ec, ej = self.ec, self.ej
        gj = g[np.where(self.ghost_nb, ec, np.minimum(ej, N - 1))]
        limj = lim[np.where(self.ghost_nb, ec, np.minimum(ej, N - 1))]
        vi = np.column_stack([self.p, self.u])[ec]
        vj = np.column_stack([self.p, self.u])[ej]
        L = vi + np.einsum("ncb,nb->nc", g[ec], self.d0) * lim[ec]
        R = vj + np.einsum("ncb,nb->nc", gj, self.d1) * limj
        n = self.n
        unL = np.einsum("ij,ij->i", L[:, 1:], n)
        unR = np.einsum("ij,ij->i", R[:, 1:], n)
        lam = np.maximum(np.abs(unL) + np.sqrt(unL ** 2 + self.beta2), np.abs(unR) + np.sqrt(unR ** 2 + self.beta2))
        h = 0.5 * self.ds
        fp = self.beta2 * (unL + unR) * h - lam * h * (R[:, 0] - L[:, 0])
        fu = ((L[:, 1:] * unL[:, None] + n * L[:, 0:1] + R[:, 1:] * unR[:, None] + n * R[:, 0:1]) * h[:, None]
              - (R[:, 1:] - L[:, 1:]) * (lam * h)[:, None])
        ga = 0.5 * (g[ec, 1:, :] + gj[:, 1:, :])                     # (S, 3 comps, 3)
        gn = np.einsum("scb,sb->sc", ga, n)
        if self.corrected:
            du = vj[:, 1:] - vi[:, 1:]
            gd = np.einsum("scb,sb->sc", ga, self.d)
            gn = gn + (du - gd) * (self.w2 * np.einsum("ij,ij->i", self.d, n))[:, None]
        fu = fu - gn * (self.nu * self.ds)[:, None]
        sr = (lam + 2.0 * self.nu * np.sqrt(self.w2)) * self.ds
        rp = self.cellsum(fp)
        ru = self.cellsum(fu)
        srs = self.cellsum(sr)
        dt = cfl / srs
        self.p[:N] -= rp * dt
        self.u[:N] -= ru * dt[:, None]
        return float(np.sum((rp ** 2 + np.einsum("ij,ij->i", ru, ru)) * self.vol[:N]))

    def run(self, bcs, n_iter, cfl):
        hist = np.zeros(n_iter)
        for k in range(n_iter):
            self.apply_bcs(bcs)
            hist[k] = self.step(cfl)
        return hist

    def wall_force(self, region):
        """density * sum over the region's faces of A (p_f n - nu G_f . n)."""
        g, _ = self.gradients()
        r = self.m.region_id(region)
        ghosts = self.gid[self.gstart[r]:self.gstart[r + 1]]
        k = ghosts - self.N
        i, n, f = self.g_int[k], self.g_n[k], self.g_face[k]
        d = self.cc[ghosts] - self.cc[i]
        w2 = 1.0 / np.einsum("ij,ij->i", d, d)
        ga = g[i, 1:, :]
        gn = np.einsum("scb,sb->sc", ga, n)
        if self.corrected:
            du = self.u[ghosts] - self.u[i]
            gn = gn + (du - np.einsum("scb,sb->sc", ga, d)) * (w2 * np.einsum("ij,ij->i", d, n))[:, None]
        pf = 0.5 * (self.p[i] + self.p[ghosts])
        return self.density * np.sum(self.area[f][:, None] * (pf[:, None] * n - self.nu * gn), axis=0)
