"""FP64 restatement of the reference's generic finite-volume operators
(include/fvmops.cuh:96-219) and of the least-squares gradient + limiter of a
field (src/fvmops.cu:51-266) -- test infrastructure only.

Every operator sums over the faces of each interior cell c0 (fvmOpSetup,
include/fvmops.cuh:33-48): c1 the neighbour, d0 = fc - x(c0), d1 = fc - x(c1),
n the normal oriented away from c0 (sign(0) = +1), ds = A / V(c0).  A ghost
neighbour carries its interior cell's gradient and limiter.  Tensors are
(u, v, w) with outer(a, b) = (a b.x, a b.y, a b.z).
"""
from __future__ import annotations

import numpy as np

from .nsi_oracle import limiter
from .pyoracle import OracleMesh


class OpMesh:
    def __init__(self, mesh: OracleMesh):
        N = mesh.N
        self.N = N
        cfs, cf, cc = mesh.get("cell_faces_starts"), mesh.get("cell_faces"), mesh.get("cell_connects")
        fn = mesh.get("face_normals").reshape(-1, 3)
        self.fc_all = mesh.get("face_centers").reshape(-1, 3)
        x = mesh.get("cell_centers").reshape(-1, 3)
        area, vol = mesh.get("face_areas"), mesh.get("cell_volumes")
        counts = np.diff(cfs[: N + 1])
        self.c0 = np.repeat(np.arange(N), counts)
        self.f = cf[cfs[0]:cfs[N]]
        self.c1 = cc[cfs[0]:cfs[N]]
        self.fc = self.fc_all[self.f]
        self.d0 = self.fc - x[self.c0]
        self.d1 = self.fc - x[self.c1]
        s = np.einsum("ij,ij->i", fn[self.f], self.d0)
        self.n = fn[self.f] * np.where(s >= 0, 1.0, -1.0)[:, None]
        self.ds = area[self.f] / vol[self.c0]
        self.g1 = np.where(self.c1 >= N, self.c0, self.c1)      # gradient owner of the neighbour
        self.dn = x[self.c1] - x[self.c0]
        self.w2 = 1.0 / np.einsum("ij,ij->i", self.dn, self.dn)
        A = np.zeros((N, 3, 3))
        np.add.at(A, self.c0, np.einsum("ij,ik->ijk", self.dn, self.dn) * self.w2[:, None, None])
        self.Ainv = np.linalg.inv(A)
        self.k3 = np.linalg.norm(self.d0, axis=1) ** 3

    def csum(self, vals):
        out = np.zeros((self.N,) + vals.shape[1:])
        np.add.at(out, self.c0, vals)
        return out

    def gradient(self, u):
        """u[(N+G), k] -> (grad[N, k, 3], lim[N, k])."""
        N = self.N
        u = u.reshape(len(u), -1)
        s = self.csum((u[self.c1] - u[self.c0])[:, :, None] * self.dn[:, None, :] * self.w2[:, None, None])
        g = np.einsum("nab,ncb->nca", self.Ainv, s)
        lo, hi = u[:N].copy(), u[:N].copy()
        np.minimum.at(lo, self.c0, u[self.c1])
        np.maximum.at(hi, self.c0, u[self.c1])
        lim = np.full(lo.shape, 2.0)
        for c in range(u.shape[1]):
            l = limiter(u[self.c0, c], g[self.c0, c], lo[self.c0, c], hi[self.c0, c], self.d0, self.k3)
            np.minimum.at(lim[:, c], self.c0, l)
        return g, lim

    def apply(self, op, u, grad=None, lim=None, phi=None, phi_c=None):
        """grad[N, k, 3], lim[N, k] as gradient() returns; phi[(N+G), 3]."""
        n, ds, d0, d1 = self.n, self.ds[:, None], self.d0, self.d1
        nrm = lambda a: np.linalg.norm(a, axis=1)
        if op in (0, 1, 2, 4, 7, 8, 9):
            u0, u1 = u[self.c0], u[self.c1]
            if op == 0:
                g = grad[:, 0, :]
                return self.csum(np.einsum("ij,ij->i", g[self.g1] + g[self.c0], n) * 0.5 * self.ds)
            if op == 1:
                phi_w = nrm(d0) / nrm(d0 - d1)
                return self.csum(n * ((u1 * phi_w + u0 * (1 - phi_w))[:, None] * ds))
            if op == 2:
                phi_w = nrm(d0) / nrm(d0 - d1)
                d_err = self.fc - (d0 - d1) * phi_w[:, None]
                return self.csum(n * (np.einsum("ij,ij->i", grad[self.c0, 0], d_err)[:, None] * ds))
            if op == 4:
                return self.csum(n * ((u1 - u0)[:, None] * ds))
            if op in (7, 8):
                a, b = u0, u1
                if op == 8:
                    a = u0 + np.einsum("ij,ij->i", grad[self.c0, 0], d0) * lim[self.c0, 0]
                    b = u1 + np.einsum("ij,ij->i", grad[self.g1, 0], d1) * lim[self.g1, 0]
                an = n @ np.asarray(phi_c, np.float64)
                return self.csum(((an * a + an * b) - np.abs(an) * (b - a)) * 0.5 * self.ds)
            a0 = np.einsum("ij,ij->i", n, phi[self.c0])
            a1 = np.einsum("ij,ij->i", n, phi[self.c1])
            return self.csum(((a0 * u0 + a1 * u1) - np.maximum(np.abs(a0), np.abs(a1)) * (u1 - u0)) * 0.5 * self.ds)
        u0, u1 = u[self.c0], u[self.c1]
        if op == 3:
            phi_w = nrm(d0) / (nrm(d0) + nrm(d1))
            w = (u1 * phi_w[:, None] + u0 * (1 - phi_w[:, None])) * ds
            return self.csum(np.einsum("si,sk->ski", n, w).reshape(-1, 9))      # column k = n * w_k
        if op == 5:
            du = (u1 - u0) * ds
            return self.csum(np.einsum("si,sk->ski", du, n).reshape(-1, 9))     # column k = du * n_k
        if op == 6:
            return self.csum(np.einsum("ij,ij->i", u0 + u1, n) * 0.5 * self.ds)
        a0 = np.einsum("ij,ij->i", n, phi[self.c0])
        a1 = np.einsum("ij,ij->i", n, phi[self.c1])
        return self.csum(((u0 * a0[:, None] + u1 * a1[:, None]) - (u1 - u0) * np.maximum(a0, a1)[:, None]) * 0.5 * ds)
