"""FP64 PyTorch restatement of the forward path, for reference gradients.
TEST INFRASTRUCTURE ONLY (the oracle): tests/ differentiate it with autograd
to check the product's hand-written discrete adjoint. It restates the same
discretisation as ns3d_oracle.c (itself pinned against the reference) with
periodic shifts (torch.roll) in place of ghost cells; a CPU test checks it
against ns3d_oracle.c.

Supported: Steger-Warming (optional entropy fix) and Lax-Friedrichs,
WENO5 and the linear reconstructions (MDCD, UPWIND_7TH, UD7L), C4/C6/C8.
State W: tensor (5, nz, ny, nx) of primitives (rho, u, v, w, p).
"""
from __future__ import annotations

import torch

# reference enum codes (field_structures.h:112-131)
WENO5, LINEAR, MDCD, UPWIND_7TH, UD7L = 0, 2, 3, 5, 6


class TorchRef:
    def __init__(self, d: dict):
        """`d` is oracle.derived(cfg)."""
        self.d = d
        self.g = d["gamma"]
        self.recon = d["recon"]
        self.S = 8 if self.recon in (UPWIND_7TH, UD7L) else (2 if self.recon == LINEAR else 6)
        self.lin = self._lin()
        self.ord = {0: 8, 1: 6, 2: 4}[d["vis"]]

    def _lin(self):
        d = self.d
        if self.recon == MDCD:
            disp, diss = d["mdcd_disp"], d["mdcd_diss"]
            return [0.5 * disp + 0.5 * diss, -1.5 * disp - 2.5 * diss - 1.0 / 12.0,
                    7.0 / 12.0 + disp + 5.0 * diss, 7.0 / 12.0 + disp - 5.0 * diss,
                    -1.5 * disp + 2.5 * diss - 1.0 / 12.0, 0.5 * disp - 0.5 * diss]
        if self.recon == UPWIND_7TH:
            return [-1 / 140, 5 / 84, -101 / 420, 319 / 420, 107 / 210, -19 / 210, 1 / 105, 0.0]
        if self.recon == UD7L:
            a = d["ud7l_alpha"]
            b = 1.0 - a
            return [-3 / 420 * a - 3 / 840 * b, 25 / 420 * a + 29 / 840 * b,
                    -101 / 420 * a - 139 / 840 * b, 319 / 420 * a + 533 / 840 * b,
                    214 / 420 * a + 533 / 840 * b, -38 / 420 * a - 139 / 840 * b,
                    4 / 420 * a + 29 / 840 * b, -3 / 840 * b]
        return None

    # -- pieces ---------------------------------------------------------------
    def _split(self, W, dim):
        g, eps = self.g, self.d["sw_eps"]
        rho, u, v, w, p = W
        vel = (u, v, w)
        un = vel[dim]
        k = 0.5 * (u * u + v * v + w * w)
        E = rho * (p / ((g - 1.0) * rho) + k)
        c = torch.sqrt(g * p / rho)
        if self.d["fvs"] == 0:
            def absf(l):
                return torch.sqrt(l * l + eps * eps) if eps > 0 else torch.abs(l)
            ls = (un - c, un, un + c)
            lp = [0.5 * (l + absf(l)) for l in ls]
            lm = [0.5 * (l - absf(l)) for l in ls]
            H = (E + p) / rho
            ga1 = rho / (2.0 * g)
            ga2 = 2.0 * (g - 1.0)
            out = []
            for L in (lp, lm):
                S1 = L[0] + L[2]
                S2 = L[2] - L[0]
                F = [ga1 * (S1 + ga2 * L[1])]
                for j in range(3):
                    term = S1 * vel[j] + ga2 * L[1] * vel[j]
                    if j == dim:
                        term = term + S2 * c
                    F.append(ga1 * term)
                F.append(ga1 * (S1 * H + ga2 * L[1] * k + S2 * un * c))
                out.append(torch.stack(F))
            return out[0], out[1]
        amax = torch.abs(un) + c
        F = [rho * un]
        for j in range(3):
            F.append(rho * vel[j] * un + (p if j == dim else 0.0 * p))
        F.append((E + p) * un)
        F = torch.stack(F)
        U = torch.stack([rho, rho * u, rho * v, rho * w, E])
        return 0.5 * (F + amax * U), 0.5 * (F - amax * U)

    def _recon(self, a):
        """a: list of S window tensors (oriented)."""
        if self.recon == WENO5:
            f0, f1, f2, f3, f4 = a[:5]
            eps = 1e-6
            b0 = 13.0 / 12.0 * (f0 - 2 * f1 + f2) ** 2 + 0.25 * (f0 - 4 * f1 + 3 * f2) ** 2
            b1 = 13.0 / 12.0 * (f1 - 2 * f2 + f3) ** 2 + 0.25 * (f1 - f3) ** 2
            b2 = 13.0 / 12.0 * (f2 - 2 * f3 + f4) ** 2 + 0.25 * (3 * f2 - 4 * f3 + f4) ** 2
            a0 = 0.1 / (eps + b0) ** 2
            a1 = 0.6 / (eps + b1) ** 2
            a2 = 0.3 / (eps + b2) ** 2
            s = a0 + a1 + a2
            p0 = (2 * f0 - 7 * f1 + 11 * f2) / 6.0
            p1 = (-f1 + 5 * f2 + 2 * f3) / 6.0
            p2 = (2 * f2 + 5 * f3 - f4) / 6.0
            return (a0 * p0 + a1 * p1 + a2 * p2) / s
        if self.recon == LINEAR:
            return a[0]
        return sum(c * x for c, x in zip(self.lin, a))

    def _dc(self, f, dim, h):
        def at(o):
            return torch.roll(f, shifts=-o, dims=dim)
        if self.ord == 4:
            return (-at(2) + 8.0 * at(1) - 8.0 * at(-1) + at(-2)) / (12.0 * h)
        if self.ord == 6:
            return (at(3) - 9.0 * at(2) + 45.0 * at(1) - 45.0 * at(-1) + 9.0 * at(-2) - at(-3)) / (
                60.0 * h)
        c1, c2, c3, c4 = 0.8, -0.2, 0.0380952380952381, -0.00357142857142857
        return (c1 * (at(1) - at(-1)) + c2 * (at(2) - at(-2)) + c3 * (at(3) - at(-3)) +
                c4 * (at(4) - at(-4))) / h

    # -- RHS and step -----------------------------------------------------------
    def rhs(self, W):
        d = self.d
        S, MID = self.S, (self.S - 1) // 2
        inv = (1.0 / d["dx"], 1.0 / d["dy"], 1.0 / d["dz"])
        tacc = None
        for dd, dim in ((0, 3), (1, 2), (2, 1)):   # x, y, z (tensor dims of (5,nz,ny,nx))
            Fp, Fm = self._split(W, dd)
            face = []
            for q in range(5):
                a = [torch.roll(Fp[q], shifts=MID - m, dims=dim - 1) for m in range(S)]
                b = [torch.roll(Fm[q], shifts=MID - S + 1 + m, dims=dim - 1) for m in range(S)]
                face.append(self._recon(a) + self._recon(b))
            face = torch.stack(face)
            diff = (face - torch.roll(face, shifts=1, dims=dim)) * inv[dd]
            tacc = diff if tacc is None else tacc + diff
        rho, u, v, w, p = W
        T = p / (rho * d["Rgas"])
        h = (d["dx"], d["dy"], d["dz"])
        dims = (2, 1, 0)  # x, y, z on (nz, ny, nx)
        grads = {}
        for name, f in (("u", u), ("v", v), ("w", w), ("T", T)):
            for a in range(3):
                grads[name + "xyz"[a]] = self._dc(f, dims[a], h[a])
        Sr = d["sutherland_s"]
        mu = d["mu"] * T ** 1.5 * (1.0 + Sr) / (T + Sr)
        div = grads["ux"] + grads["vy"] + grads["wz"]
        txx = 2.0 * mu * grads["ux"] - 2.0 / 3.0 * mu * div
        tyy = 2.0 * mu * grads["vy"] - 2.0 / 3.0 * mu * div
        tzz = 2.0 * mu * grads["wz"] - 2.0 / 3.0 * mu * div
        txy = mu * (grads["uy"] + grads["vx"])
        txz = mu * (grads["uz"] + grads["wx"])
        tyz = mu * (grads["vz"] + grads["wy"])
        kq = mu * d["Cp"] / d["Pr"]
        ex = u * txx + v * txy + w * txz + kq * grads["Tx"]
        ey = u * txy + v * tyy + w * tyz + kq * grads["Ty"]
        ez = u * txz + v * tyz + w * tzz + kq * grads["Tz"]
        Fv = (txx, txy, txz, ex)
        Hv = (txy, tyy, tyz, ey)
        Gv = (txz, tyz, tzz, ez)
        vis = [torch.zeros_like(u)]
        for m in range(4):
            vis.append(self._dc(Fv[m], 2, h[0]) + self._dc(Hv[m], 1, h[1]) +
                       self._dc(Gv[m], 0, h[2]))
        return torch.stack(vis) - tacc

    def p2c(self, W):
        g = self.g
        rho, u, v, w, p = W
        k = 0.5 * (u * u + v * v + w * w)
        return torch.stack([rho, rho * u, rho * v, rho * w, rho * (p / ((g - 1.0) * rho) + k)])

    def c2p(self, U):
        g = self.g
        rho = U[0]
        u, v, w = U[1] / rho, U[2] / rho, U[3] / rho
        k = 0.5 * (u * u + v * v + w * w)
        p = (g - 1.0) * rho * (U[4] / rho - k)
        return torch.stack([rho, u, v, w, p])

    def rk3(self, W, dt):
        U0 = self.p2c(W)
        W1 = self.c2p(U0 + dt * self.rhs(W))
        W2 = self.c2p(0.75 * U0 + 0.25 * (self.p2c(W1) + dt * self.rhs(W1)))
        return self.c2p(1.0 / 3.0 * U0 + 2.0 / 3.0 * (self.p2c(W2) + dt * self.rhs(W2)))

    def kinetic_energy(self, W):
        d = self.d
        rho, u, v, w = W[0], W[1], W[2], W[3]
        return (0.5 * rho * (u * u + v * v + w * w)).sum() * (d["dx"] * d["dy"] * d["dz"])
