"""CPU restatement of the surrogate network (test infrastructure only).

The reference has no learned component; this file is the oracle for the
project's own Fourier neural operator (scattersim_b200/csrc/fno.cu): the same
parameter layout, the same separable DFT operators, and the same arithmetic
points -- every GEMM rounds its two operands to BF16 (round to nearest even)
and accumulates in float64 here (float32 on the GPU), and every stored
intermediate is float32.  With ``bf16=False`` the network runs in float64
throughout, which the finite-difference tests use to pin the backward pass.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

G = 64
NP = G * G
W = 64
CIN = 6
SLAB_UM = 1.0
L = 4
MX = MY = 16
NM = 2 * MX * MY
NF = 2 * NM
HID = 128
COUT = 12
NO = 11
NORD = NO * NO
NOUT = 6 * NORD * 2


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


class Layout:
    """Offsets of the flat parameter vector (fno.cu::Layout, 64-float aligned blocks)."""

    def __init__(self):
        self.o = 0

        def take(n):
            r = self.o
            self.o += (n + 63) // 64 * 64
            return r
        self.P = take(W * CIN)
        self.bP = take(W)
        self.Wl, self.bl, self.SWr, self.SWi = [], [], [], []
        for _ in range(L):
            self.Wl.append(take(W * W))
            self.bl.append(take(W))
            self.SWr.append(take(NM * W * W))
            self.SWi.append(take(NM * W * W))
        self.Q1 = take(HID * W)
        self.bQ1 = take(HID)
        self.Q2 = take(COUT * HID)
        self.bQ2 = take(COUT)
        self.total = self.o


def kx_of(r):
    return r if r < MX else r - 2 * MX


def operators():
    """Separable DFT operators and the readout, as fno.cu::build_operators.

    Fy (64 x 32), Ex (64 x 64), Er (64 x 64), Ei (64 x 64), Gy (32 x 64), R (NP x 2 NORD).
    """
    tp = 2 * np.pi / G

    def trig(ph):
        th = tp * ((np.asarray(ph) % G + G) % G)
        return np.cos(th), np.sin(th)
    y = np.arange(G)
    ky = np.arange(MY)
    c, s_ = trig(np.outer(y, ky))                       # (y, ky)
    Fy = np.concatenate([c, -s_], axis=1)
    cw = np.where(ky == 0, 1.0, 2.0)[:, None] / NP
    Gy = np.concatenate([cw * c.T, -cw * s_.T], axis=0)   # (32, y)
    kx = np.array([kx_of(r) for r in range(2 * MX)])
    x = np.arange(G)
    c, s_ = trig(np.outer(kx, x))                         # (r, x)
    Ex = np.concatenate([c, s_], axis=0)                  # (64 rows, x)
    Er = np.concatenate([c.T, -s_.T], axis=1)             # (x, 64)
    Ei = np.concatenate([s_.T, c.T], axis=1)
    R = np.zeros((NP, 2 * NORD))
    xx = np.repeat(np.arange(G), G)
    yy = np.tile(np.arange(G), G)
    for j in range(NORD):
        qq = j % NO - NO // 2
        pp = j // NO - NO // 2
        cc, ss = trig(pp * xx + qq * yy)
        R[:, j] = cc / NP
        R[:, NORD + j] = ss / NP
    return tuple(a.astype(np.float32) for a in (Fy, Ex, Er, Ei, Gy, R))


class Net:
    def __init__(self, params, bf16_ops=True):
        self.lay = Layout()
        self.w = np.asarray(params, dtype=np.float32)
        self.q = bf16_ops
        self.Fy, self.Ex, self.Er, self.Ei, self.Gy, self.R = operators()
        self.dt = np.float32 if bf16_ops else np.float64
        if not bf16_ops:
            self.w = self.w.astype(np.float64)
            self.Fy, self.Ex, self.Er, self.Ei, self.Gy, self.R = (
                a.astype(np.float64) for a in (self.Fy, self.Ex, self.Er, self.Ei, self.Gy, self.R))

    # a GEMM the way the GPU does it: BF16 operands, wide accumulation, stored as float32
    def mm(self, A, B):
        if self.q:
            out = bf16(A).astype(np.float64) @ bf16(B).astype(np.float64)
            return out.astype(np.float32)
        return A @ B

    def bmm(self, A, B):
        """Batched GEMM (broadcast leading dims), same arithmetic as mm."""
        if self.q:
            return np.matmul(bf16(A).astype(np.float64), bf16(B).astype(np.float64)).astype(np.float32)
        return np.matmul(A, B)

    def fwd_dft(self, v):
        """v (B, W, NP) -> X (B, W, NF): along y, then x, combined (fno.cu)."""
        B = v.shape[0]
        A1 = self.mm(v.reshape(-1, G), self.Fy).reshape(B * W, G, 2 * MY)
        U = self.bmm(self.Ex[None], A1)                                     # (nch, 64, 32)
        X = np.zeros((B * W, NF), self.dt)
        r, ky = np.divmod(np.arange(NM), MY)
        X[:, :NM] = (U[:, r, ky] + U[:, 2 * MX + r, MY + ky]).astype(self.dt)
        X[:, NM:] = (U[:, r, MY + ky] - U[:, 2 * MX + r, ky]).astype(self.dt)
        return X.reshape(B, W, NF)

    def inv_dft(self, Y):
        """Y (B, W, NF) -> the spectral branch of u (B, W, NP)."""
        B = Y.shape[0]
        Yc = Y.reshape(B * W, G, MY)                                          # rows: [re r | im r]
        Z = np.concatenate([self.bmm(self.Er[None], Yc), self.bmm(self.Ei[None], Yc)], axis=2)   # (nch, 64, 32)
        return self.mm(Z.reshape(-1, 2 * MY), self.Gy).reshape(B, W, NP)

    def fwd_dft_adj(self, dX):
        """Adjoint of fwd_dft: dX (B, W, NF) -> dv (B, W, NP)."""
        B = dX.shape[0]
        dXc = dX.reshape(B * W, NF)
        dU = np.zeros((B * W, G, 2 * MY), self.dt)
        r, ky = np.divmod(np.arange(NM), MY)
        dU[:, r, ky] = dXc[:, :NM]
        dU[:, 2 * MX + r, MY + ky] = dXc[:, :NM]
        dU[:, r, MY + ky] = dXc[:, NM:]
        dU[:, 2 * MX + r, ky] = -dXc[:, NM:]
        dA1 = self.bmm(self.Ex.T[None], dU)
        return self.mm(dA1.reshape(-1, 2 * MY), self.Fy.T).reshape(B, W, NP)

    def inv_dft_adj(self, du):
        """Adjoint of inv_dft: du (B, W, NP) -> dY (B, W, NF)."""
        B = du.shape[0]
        dZ = self.mm(du.reshape(-1, G), self.Gy.T).reshape(B * W, G, 2 * MY)
        dY = (self.bmm(self.Er.T[None], dZ[:, :, :MY]).astype(np.float64)
              + self.bmm(self.Ei.T[None], dZ[:, :, MY:]).astype(np.float64)).astype(self.dt)
        return dY.reshape(B, W, NF)

    def par(self, off, shape):
        n = int(np.prod(shape))
        return self.w[off:off + n].reshape(shape)

    def gelu(self, x):
        return (0.5 * x * (1.0 + erf(x.astype(np.float64) / np.sqrt(2.0)))).astype(self.dt)

    def gelu_grad(self, x):
        xd = x.astype(np.float64)
        return (0.5 * (1.0 + erf(xd / np.sqrt(2.0))) + xd * np.exp(-0.5 * xd * xd) / np.sqrt(2 * np.pi)).astype(self.dt)

    def forward(self, maps, lam):
        Ly = self.lay
        B = maps.shape[0]
        c = {}
        inp = np.zeros((B, CIN, NP), self.dt)
        inp[:, 0] = maps.reshape(B, NP)
        inp[:, 1] = ((np.asarray(lam, np.float32) - np.float32(0.6)) / np.float32(0.2))[:, None]
        p = np.arange(NP)
        inp[:, 2] = (p // G).astype(np.float32) / np.float32(63)
        inp[:, 3] = (p % G).astype(np.float32) / np.float32(63)
        # thin-element phase of the slab, in turns reduced to [0, 1) in float32
        turns = (np.asarray(maps, np.float32).reshape(B, NP) * np.float32(SLAB_UM)
                 / np.asarray(lam, np.float32)[:, None]).astype(np.float32)
        fr = (turns - np.floor(turns)).astype(np.float32)
        inp[:, 4] = np.cos(2 * np.pi * fr.astype(np.float64)).astype(np.float32)
        inp[:, 5] = np.sin(2 * np.pi * fr.astype(np.float64)).astype(np.float32)
        c["in"] = inp
        P = self.par(Ly.P, (W, CIN))
        v = np.stack([self.mm(P, inp[b]) for b in range(B)]) + self.par(Ly.bP, (W,))[None, :, None]
        v = v.astype(self.dt)
        acts, pres, Xs = [v], [], []
        for l in range(L):
            X = self.fwd_dft(v)                                                   # B x W x NF
            Xs.append(X)
            Wr = self.par(Ly.SWr[l], (NM, W, W))
            Wi = self.par(Ly.SWi[l], (NM, W, W))
            Xr, Xi = X[:, :, :NM], X[:, :, NM:]
            Y = np.zeros_like(X)
            for md in range(NM):
                a, bm = Xr[:, :, md], Xi[:, :, md]
                Y[:, :, md] = (self.mm(a, Wr[md]).astype(np.float64) - self.mm(bm, Wi[md]).astype(np.float64)).astype(self.dt)
                Y[:, :, NM + md] = (self.mm(a, Wi[md]).astype(np.float64) + self.mm(bm, Wr[md]).astype(np.float64)).astype(self.dt)
            Wl = self.par(Ly.Wl[l], (W, W))
            u = np.stack([self.mm(Wl, v[b]) for b in range(B)])
            u = (u.astype(np.float64) + self.inv_dft(Y).astype(np.float64)).astype(self.dt)
            u = (u + self.par(Ly.bl[l], (W,))[None, :, None]).astype(self.dt)
            pres.append(u)
            v = self.gelu(u) if l < L - 1 else u
            acts.append(v)
        Q1 = self.par(Ly.Q1, (HID, W))
        hpre = (np.stack([self.mm(Q1, v[b]) for b in range(B)]) + self.par(Ly.bQ1, (HID,))[None, :, None]).astype(self.dt)
        h = self.gelu(hpre)
        Q2 = self.par(Ly.Q2, (COUT, HID))
        o = (np.stack([self.mm(Q2, h[b]) for b in range(B)]) + self.par(Ly.bQ2, (COUT,))[None, :, None]).astype(self.dt)
        Pc = np.stack([self.mm(o[b], self.R) for b in range(B)])             # B x 12 x 242
        pred = np.zeros((B, 6, NORD, 2), self.dt)
        for ch in range(6):
            pr, pi = Pc[:, 2 * ch], Pc[:, 2 * ch + 1]
            pred[:, ch, :, 0] = pr[:, :NORD] + pi[:, NORD:]
            pred[:, ch, :, 1] = pi[:, :NORD] - pr[:, NORD:]
        c.update(acts=acts, pres=pres, Xs=Xs, hpre=hpre, h=h, o=o)
        self.cache = c
        return pred.reshape(B, NOUT)

    def loss_grad(self, maps, lam, target):
        """Mean relative squared error and its gradient (flat, like the parameters)."""
        Ly = self.lay
        pred = self.forward(maps, lam)
        c = self.cache
        B = pred.shape[0]
        tgt = np.asarray(target, self.dt)
        d = pred.astype(np.float64) - tgt
        nrm = (tgt.astype(np.float64) ** 2).sum(1)
        loss = (d ** 2).sum(1) / nrm
        dpred = (2.0 * d / (nrm[:, None] * B)).astype(self.dt).reshape(B, 6, NORD, 2)
        g = np.zeros(Ly.total, np.float64)

        def acc(off, val):
            g[off:off + val.size] += val.ravel()

        dP = np.zeros((B, COUT, 2 * NORD), self.dt)
        for ch in range(6):
            dP[:, 2 * ch, :NORD] = dpred[:, ch, :, 0]
            dP[:, 2 * ch + 1, NORD:] = dpred[:, ch, :, 0]
            dP[:, 2 * ch + 1, :NORD] = dpred[:, ch, :, 1]
            dP[:, 2 * ch, NORD:] = -dpred[:, ch, :, 1]
        do = np.stack([self.mm(dP[b], self.R.T) for b in range(B)])
        acc(Ly.Q2, sum(self.mm(do[b], c["h"][b].T).astype(np.float64) for b in range(B)))
        acc(Ly.bQ2, do.astype(np.float64).sum((0, 2)))
        Q2 = self.par(Ly.Q2, (COUT, HID))
        dh = np.stack([self.mm(Q2.T, do[b]) for b in range(B)])
        dh = (dh * self.gelu_grad(c["hpre"])).astype(self.dt)
        acc(Ly.Q1, sum(self.mm(dh[b], c["acts"][L][b].T).astype(np.float64) for b in range(B)))
        acc(Ly.bQ1, dh.astype(np.float64).sum((0, 2)))
        Q1 = self.par(Ly.Q1, (HID, W))
        dv = np.stack([self.mm(Q1.T, dh[b]) for b in range(B)])
        for l in range(L - 1, -1, -1):
            du = dv if l == L - 1 else (dv * self.gelu_grad(c["pres"][l])).astype(self.dt)
            acc(Ly.bl[l], du.astype(np.float64).sum((0, 2)))
            vin = c["acts"][l]
            acc(Ly.Wl[l], sum(self.mm(du[b], vin[b].T).astype(np.float64) for b in range(B)))
            Wl = self.par(Ly.Wl[l], (W, W))
            dvn = np.stack([self.mm(Wl.T, du[b]) for b in range(B)])
            dY = self.inv_dft_adj(du)
            X = c["Xs"][l]
            Xr, Xi = X[:, :, :NM], X[:, :, NM:]
            dYr, dYi = dY[:, :, :NM], dY[:, :, NM:]
            Wr = self.par(Ly.SWr[l], (NM, W, W))
            Wi = self.par(Ly.SWi[l], (NM, W, W))
            dX = np.zeros_like(X)
            gWr = np.zeros((NM, W, W))
            gWi = np.zeros((NM, W, W))
            for md in range(NM):
                r, i = dYr[:, :, md], dYi[:, :, md]
                dX[:, :, md] = (self.mm(r, Wr[md].T).astype(np.float64) + self.mm(i, Wi[md].T).astype(np.float64)).astype(self.dt)
                dX[:, :, NM + md] = (-self.mm(r, Wi[md].T).astype(np.float64) + self.mm(i, Wr[md].T).astype(np.float64)).astype(self.dt)
                xr, xi = Xr[:, :, md], Xi[:, :, md]
                gWr[md] = self.mm(xr.T, r).astype(np.float64) + self.mm(xi.T, i).astype(np.float64)
                gWi[md] = -self.mm(xi.T, r).astype(np.float64) + self.mm(xr.T, i).astype(np.float64)
            acc(Ly.SWr[l], gWr)
            acc(Ly.SWi[l], gWi)
            dv = (dvn.astype(np.float64) + self.fwd_dft_adj(dX).astype(np.float64)).astype(self.dt)
        acc(Ly.P, sum(self.mm(dv[b], c["in"][b].T).astype(np.float64) for b in range(B)))
        acc(Ly.bP, dv.astype(np.float64).sum((0, 2)))
        return loss, g
