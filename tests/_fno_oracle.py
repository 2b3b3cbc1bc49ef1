"""FP64 numpy restatement of the learned warm start (isg_fno.cu): the same
network, parameter layout and loss, with a hand-written backward pass.  Test
infrastructure only: it checks the CUDA kernels' outputs and gradients, and is
itself checked against finite differences.

Network per sample (raster order, N x N pixels, width C, L layers, M kx modes,
KY = 2M ky modes: ky in [0, M) and [N - M, N)):
  in   = [chi, b, chi b, s1, chi s1] as (Re, Im) pairs, chi = g / k0^2,
         s1 = G(g b) the first Born scattered field (given)
  v0   = Wl in + bl
  h_l  = W_l v_l + bw_l + spec_l(v_l),  v_{l+1} = gelu(h_l) (identity after the last layer)
  spec = (T -> X -> Y -> Z -> spec):  T = v Ex (DFT along x, kx < M),
         X = Fy T (DFT along y), Y[o] = sum_c R[k,o,c] X[c], Z = Fy^H Y,
         spec = Z Ix (real part of the inverse DFT along x, weight 2 for kx > 0, / N^2)
  pred = b + (Wp v_L + Ws in + bp)_0 + i (Wp v_L + Ws in + bp)_1
  loss = mean_s |pred_s - u_s|^2 / |u_s|^2
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


NIN = 10


def layout(C: int, M: int, L: int):
    """Offsets of the flat parameter vector (each block on a 4-float boundary)."""
    NM = 2 * M * M
    off = 0
    out = {}

    def take(name, n):
        nonlocal off
        out[name] = (off, n)
        off += (n + 3) // 4 * 4

    take("Wl", C * NIN)
    take("bl", C)
    for l in range(L):
        take(f"R{l}", 2 * NM * C * C)
        take(f"W{l}", C * C)
        take(f"bw{l}", C)
    take("Wp", 2 * C)
    take("Ws", 2 * NIN)
    take("bp", 2)
    return out, off


class FnoOracle:
    def __init__(self, N: int, C: int, M: int, L: int, k0: float = 2 * math.pi):
        self.N, self.C, self.M, self.L, self.k0 = N, C, M, L, k0
        self.KY, self.NM = 2 * M, 2 * M * M
        self.lay, self.nparam = layout(C, M, L)
        th = 2 * math.pi / N
        x = np.arange(N)
        k = np.arange(M)
        a = th * ((k[None, :] * x[:, None]) % N)
        self.Ex = np.zeros((N, 2 * M))
        self.Ex[:, 0::2] = np.cos(a)
        self.Ex[:, 1::2] = -np.sin(a)
        w = np.where(k == 0, 1.0, 2.0) / (N * N)
        self.Ix = np.zeros((2 * M, N))
        self.Ix[0::2, :] = (w[None, :] * np.cos(a)).T
        self.Ix[1::2, :] = (-w[None, :] * np.sin(a)).T
        f = np.array([r if r < M else N - self.KY + r for r in range(self.KY)])
        self.Fy = np.exp(-1j * th * ((f[:, None] * x[None, :]) % N))  # [KY][N]

    def unpack(self, p: np.ndarray) -> dict:
        C, NM = self.C, self.NM
        d = {}
        for name, (o, n) in self.lay.items():
            v = np.asarray(p[o:o + n], dtype=np.float64)
            if name.startswith("R"):
                v = (v[0::2] + 1j * v[1::2]).reshape(NM, C, C)
            elif name == "Wl":
                v = v.reshape(C, NIN)
            elif name == "Ws":
                v = v.reshape(2, NIN)
            elif name.startswith("W") and name != "Wp":
                v = v.reshape(C, C)
            elif name == "Wp":
                v = v.reshape(2, C)
            d[name] = v
        return d

    def pack(self, d: dict) -> np.ndarray:
        p = np.zeros(self.nparam)
        for name, (o, n) in self.lay.items():
            v = d[name]
            if name.startswith("R"):
                flat = np.zeros(n)
                z = v.reshape(-1)
                flat[0::2], flat[1::2] = z.real, z.imag
                p[o:o + n] = flat
            else:
                p[o:o + n] = np.asarray(v, dtype=np.float64).reshape(-1)
        return p

    # ---- one sample ----
    def _spec(self, v, R):
        C, N, M = self.C, self.N, self.M
        T = v.reshape(C, N, N) @ self.Ex                      # (C, y, 2M)
        Tc = T[..., 0::2] + 1j * T[..., 1::2]                 # (C, y, M)
        X = np.einsum("ry,cyk->crk", self.Fy, Tc).reshape(C, -1)   # (C, NM)
        Y = np.einsum("koc,ck->ok", R, X)
        Z = np.einsum("ry,ork->oyk", self.Fy.conj(), Y.reshape(C, self.KY, M))
        Zr = np.zeros((C, N, 2 * M))
        Zr[..., 0::2], Zr[..., 1::2] = Z.real, Z.imag
        return (Zr @ self.Ix).reshape(C, N * N), X

    def forward(self, p, g, b, s1):
        """g, b, s1: complex raster vectors of one sample.  Returns (pred, cache)."""
        d = self.unpack(p)
        chi = g / self.k0 ** 2
        feats = [chi, b, chi * b, s1, chi * s1]
        inp = np.stack([f for z in feats for f in (z.real, z.imag)])
        v = d["Wl"] @ inp + d["bl"][:, None]
        vs, hs, Xs = [v], [], []
        for l in range(self.L):
            spec, X = self._spec(v, d[f"R{l}"])
            h = d[f"W{l}"] @ v + d[f"bw{l}"][:, None] + spec
            v = 0.5 * h * (1 + erf(h / math.sqrt(2))) if l + 1 < self.L else h
            hs.append(h)
            Xs.append(X)
            vs.append(v)
        out = d["Wp"] @ v + d["Ws"] @ inp + d["bp"][:, None]
        return b + out[0] + 1j * out[1], (d, inp, vs, hs, Xs)

    def backward(self, cache, dout) -> dict:
        """Parameter gradients for d loss / d out = dout (2, P) of one sample."""
        C, N, M = self.C, self.N, self.M
        d, inp, vs, hs, Xs = cache
        grads = {k: np.zeros_like(v) for k, v in d.items()}
        grads["Wp"] += dout @ vs[-1].T
        grads["Ws"] += dout @ inp.T
        grads["bp"] += dout.sum(axis=1)
        dv = d["Wp"].T @ dout
        for l in range(self.L - 1, -1, -1):
            h = hs[l]
            if l + 1 < self.L:
                dv = dv * (0.5 * (1 + erf(h / math.sqrt(2))) + h * np.exp(-0.5 * h * h) / math.sqrt(2 * math.pi))
            grads[f"bw{l}"] += dv.sum(axis=1)
            grads[f"W{l}"] += dv @ vs[l].T
            dZr = dv.reshape(C, N, N) @ self.Ix.T          # (C, y, 2M)
            dZ = dZr[..., 0::2] + 1j * dZr[..., 1::2]
            dY = np.einsum("ry,oyk->ork", self.Fy, dZ).reshape(C, -1)
            grads[f"R{l}"] += np.einsum("ok,ck->koc", dY, Xs[l].conj())
            dX = np.einsum("koc,ok->ck", d[f"R{l}"].conj(), dY)
            dT = np.einsum("ry,crk->cyk", self.Fy.conj(), dX.reshape(C, self.KY, M))
            dTr = np.zeros((C, N, 2 * M))
            dTr[..., 0::2], dTr[..., 1::2] = dT.real, dT.imag
            dv = (dTr @ self.Ex.T).reshape(C, N * N) + d[f"W{l}"].T @ dv
        grads["Wl"] += dv @ inp.T
        grads["bl"] += dv.sum(axis=1)
        return grads

    def loss_grad(self, p, G, B, S1, U):
        """Mean relative squared field error over samples and its gradient (flat)."""
        ns = len(B)
        total = None
        loss = 0.0
        for s in range(ns):
            g = G[s] if G.ndim == 2 else G
            pred, cache = self.forward(p, g, B[s], S1[s])
            e = pred - U[s]
            uu = np.vdot(U[s], U[s]).real
            loss += np.vdot(e, e).real / uu / ns
            gr = self.backward(cache, np.stack([e.real, e.imag]) * (2.0 / (uu * ns)))
            total = gr if total is None else {k: total[k] + gr[k] for k in total}
        return loss, self.pack(total)

    def residual_loss_grad(self, p, G, B, apply_A, apply_AH):
        """Mean relative squared initial residual |b - A x0|^2 / |b|^2 and its
        gradient; apply_A / apply_AH map (raster x, raster g) to raster vectors."""
        ns = len(B)
        total = None
        loss = 0.0
        for s in range(ns):
            g = G[s] if G.ndim == 2 else G
            pred, cache = self.forward(p, g, B[s], B[s] - apply_A(B[s], g))
            r = apply_A(pred, g) - B[s]
            bb = np.vdot(B[s], B[s]).real
            loss += np.vdot(r, r).real / bb / ns
            dx = apply_AH(r, g) * (2.0 / (bb * ns))
            gr = self.backward(cache, np.stack([dx.real, dx.imag]))
            total = gr if total is None else {k: total[k] + gr[k] for k in total}
        return loss, self.pack(total)

    def loss(self, p, G, B, S1, U):
        ns = len(B)
        total = 0.0
        for s in range(ns):
            g = G[s] if G.ndim == 2 else G
            pred, _ = self.forward(p, g, B[s], S1[s])
            e = pred - U[s]
            total += np.vdot(e, e).real / np.vdot(U[s], U[s]).real / ns
        return total
