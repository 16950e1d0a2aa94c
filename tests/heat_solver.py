"""Test-only harness: a time-stepped periodic reaction-diffusion solver built on
the box FGT, the way the reference's hpots solvers use boxfgt
(hpots/hpots2dadap.f: the initial-value potential with delta = 4 dt, and the
volume potential over [t_n, t_{n+1}] with one transform per time node,
delta = 4 (t_{n+1} - s)).

    u_t = Laplacian(u) + F(u, x, t),   F = S(x, t) - u^3,  periodic unit box,
    u^{n+1} = G_dt * u^n + int_{t_n}^{t_{n+1}} G_{t_{n+1}-s} * F(s) ds,
    G_tau * f = boxfgt(f, delta = 4 tau) / (4 pi tau),

with F(s) at 4 Gauss-Legendre nodes extrapolated from F^n..F^{n-3}
(4th-order Adams-Bashforth).  The 5 transforms of a step are one batch
(bfgt_batch_*), captured once as a CUDA graph and replayed every step.

Gradient of J = 0.5 |u^N - g|^2 with respect to u^0: adjoint stepping with
checkpoints every `ckpt` steps; the forward states of a segment are recomputed
from its checkpoint (the step is nonlinear through u^3), and the transposes of a
step's 5 transforms are one batched adjoint (bfgt_batch_execute_adjoint).
"""
from __future__ import annotations

import math

import numpy as np
import torch

import heat2d_per_box_b200 as hb

NQ = 4
XQ, WQ = np.polynomial.legendre.leggauss(NQ)
XQ = (XQ + 1) / 2          # nodes in (0, 1): s_q = t_n + XQ dt
WQ = WQ / 2


def ab4_weights(x):
    """Lagrange weights of the nodes t_n - j dt (j = 0..3) at t_n + x dt."""
    w = []
    for j in range(4):
        v = 1.0
        for m in range(4):
            if m != j:
                v *= (x + m) / (m - j)
        w.append(v)
    return w


class HeatStepper:
    def __init__(self, tree, dt, eps, precision, source):
        """source(t) -> S(x, t) as a device tensor in the leaf layout."""
        self.tree, self.dt, self.source = tree, dt, source
        self.tau = [(1 - x) * dt for x in XQ]
        deltas = [4 * dt] + [4 * t for t in self.tau]
        self.plans = [hb.Plan(tree, d, eps, precision=precision) for d in deltas]
        self.batch = hb.Batch(self.plans)
        off = self.batch.offsets
        self.off = off
        self.m = int(off[1])
        dev = torch.device("cuda")
        self.fin = torch.zeros(int(off[-1]), dtype=torch.float64, device=dev)
        self.pout = torch.zeros_like(self.fin)
        self.stream = torch.cuda.current_stream()
        self.batch.graph_capture(self.fin, self.pout, self.stream)
        self.lw = [ab4_weights(x) for x in XQ]
        leaf = np.zeros((tree.nboxes, tree.npbox))
        leaf[tree.leaves()] = 1.0
        self.leaf = torch.from_numpy(leaf.reshape(-1)).to(dev)
        self.c0 = 1.0 / (4 * math.pi * dt)
        self.cq = [WQ[q] * dt / (4 * math.pi * self.tau[q]) for q in range(NQ)]

    def forcing(self, u, t):
        return (self.source(t) - u ** 3) * self.leaf

    def step(self, u, fh):
        """u^{n+1} from u^n and the forcing history fh = [F^n, F^{n-1}, F^{n-2}, F^{n-3}]."""
        m = self.m
        self.fin[:m] = u
        for q in range(NQ):
            self.fin[(q + 1) * m:(q + 2) * m] = sum(self.lw[q][j] * fh[j] for j in range(4))
        self.pout.zero_()
        self.batch.graph_launch(self.stream)
        out = self.c0 * self.pout[:m]
        for q in range(NQ):
            out = out + self.cq[q] * self.pout[(q + 1) * m:(q + 2) * m]
        return out

    def run(self, u0, hist0, nsteps, keep=None):
        """hist0 = [F^{-1}, F^{-2}, F^{-3}] (fixed start-up history).  Returns u^N
        and, if keep is a dict, the windows (u^n, F^n, F^{n-1}, F^{n-2}, F^{n-3})
        at the steps it names."""
        u = u0
        fh = [self.forcing(u0, 0.0)] + list(hist0)
        for n in range(nsteps):
            if keep is not None and n in keep:
                keep[n] = (u.clone(), [f.clone() for f in fh])
            un = self.step(u, fh)
            u = un
            fh = [self.forcing(u, (n + 1) * self.dt)] + fh[:3]
        return u

    def adjoint_all(self, lam):
        """[K_k^T lam for every transform k of the step] by one batched adjoint."""
        m = self.m
        pin = lam.repeat(NQ + 1)
        out = torch.zeros_like(pin)
        self.batch.execute_adjoint(pin, out, self.stream)
        return [out[k * m:(k + 1) * m] for k in range(NQ + 1)]

    def adjoint_apply(self, k, lam):
        """K_k^T lam for transform k of the batch (0: the initial-value one)."""
        out = torch.zeros_like(lam)
        self.plans[k].execute_adjoint(lam.contiguous(), out, self.stream)
        return out

    def gradient(self, u0, hist0, nsteps, g, ckpt=20):
        """dJ/du0 for J = 0.5 |u^N - g|^2 by checkpointed adjoint stepping."""
        marks = {n: None for n in range(0, nsteps, ckpt)}
        uN = self.run(u0, hist0, nsteps, keep=marks)
        # lam[j]: dJ/du^{n+1-j} still to be propagated (j = 0 is the newest state)
        lam = [(uN - g) * self.leaf, torch.zeros_like(u0), torch.zeros_like(u0), torch.zeros_like(u0)]
        starts = sorted(marks)
        for s0 in reversed(starts):
            s1 = min(s0 + ckpt, nsteps)
            # recompute the segment's forward windows from its checkpoint
            u, fh = marks[s0]
            wins = []
            for n in range(s0, s1):
                wins.append((u, fh))
                u = self.step(u, fh)
                fh = [self.forcing(u, (n + 1) * self.dt)] + fh[:3]
            for n in reversed(range(s0, s1)):
                un, fh = wins[n - s0]
                l1 = lam[0]  # dJ/du^{n+1}
                kt = self.adjoint_all(l1)  # K_k^T l1 for the 5 transforms of the step, one batch
                gu = self.c0 * kt[0]
                wq = [self.cq[q] * kt[q + 1] for q in range(NQ)]
                # u^{n+1} depends on u^n directly and on F^{n-j}(u^{n-j}), j = 0..3
                new = [torch.zeros_like(u0) for _ in range(4)]
                new[0] = gu
                for j in range(4):
                    if n - j < 0:
                        break   # the start-up history does not depend on u0
                    uj = un if j == 0 else wins[n - s0 - j][0] if n - j >= s0 else None
                    if uj is None:
                        uj = self._state(marks, starts, n - j)
                    dF = -3.0 * uj * uj * self.leaf
                    new[j] = new[j] + dF * sum(self.lw[q][j] * wq[q] for q in range(NQ))
                lam = [lam[1] + new[0], lam[2] + new[1], lam[3] + new[2], new[3]]
        return lam[0]

    def _state(self, marks, starts, k):
        """u^k for a k before the current segment (recomputed from its checkpoint)."""
        s0 = max(s for s in starts if s <= k)
        u, fh = marks[s0]
        for n in range(s0, k):
            u2 = self.step(u, fh)
            fh = [self.forcing(u2, (n + 1) * self.dt)] + fh[:3]
            u = u2
        return u

    def close(self):
        self.batch.close()
        for p in self.plans:
            p.close()
