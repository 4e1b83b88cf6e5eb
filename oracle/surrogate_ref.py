"""CPU reference of the surrogate network -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, the forward and backward pass that gg_surrogate.cu runs on
the GPU (network definition in include/gg.h, gg_surrogate_*), so that the GPU
gradients can be checked against it.  Every matrix product rounds both operands
to bf16 (round to nearest even), as the GPU kernel does when it stages them in
shared memory; the products accumulate in float64 here (fp32 on the GPU).
`bf16=False` gives the plain float64 network for finite-difference checks of
this restatement itself.
"""
from __future__ import annotations

import numpy as np

H = 64
Z = 3 * H
LAYERS = 3


def to_bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def layout(F):
    o = {}
    k = 0
    o["win"] = (k, (F, H)); k += F * H
    o["bin"] = (k, (H,)); k += H
    for l in range(LAYERS):
        o[f"ws{l}"] = (k, (H, H)); k += H * H
        o[f"wn{l}"] = (k, (H, H)); k += H * H
        o[f"b{l}"] = (k, (H,)); k += H
    o["wr1"] = (k, (Z, H)); k += Z * H
    o["br1"] = (k, (H,)); k += H
    o["wr2"] = (k, (H,)); k += H
    o["br2"] = (k, (1,)); k += 1
    return o, k


def unpack(p, F):
    o, _ = layout(F)
    return {name: np.asarray(p[off:off + int(np.prod(shape))], dtype=np.float64).reshape(shape)
            for name, (off, shape) in o.items()}


def pack(d, F):
    o, k = layout(F)
    p = np.zeros(k, dtype=np.float64)
    for name, (off, shape) in o.items():
        p[off:off + int(np.prod(shape))] = d[name].reshape(-1)
    return p


class Net:
    def __init__(self, adj, X, bf16=True):
        self.adj = np.asarray(adj, dtype=np.int64)
        self.X = np.asarray(X, dtype=np.float64)
        self.F = self.X.shape[1]
        self.r = to_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))

    def mm(self, A, B):
        return self.r(A) @ self.r(B)

    def nbr_mean(self, Hm):
        return Hm[self.adj].mean(axis=1)

    def forward(self, p, swaps):
        W = unpack(p, self.F)
        c = {}
        h = np.maximum(self.mm(self.X, W["win"]) + W["bin"], 0)
        c["H"] = [h]
        c["M"] = []
        for l in range(LAYERS):
            m = self.nbr_mean(h)
            h = np.maximum(self.mm(h, W[f"ws{l}"]) + self.mm(m, W[f"wn{l}"]) + W[f"b{l}"], 0)
            c["M"].append(m)
            c["H"].append(h)
        a, b, cc, d = (swaps[k].astype(np.int64) for k in "abcd")
        mode = swaps["mode"]
        pp = np.where(mode == 0, cc, d)
        qq = np.where(mode == 0, d, cc)
        Hl = c["H"][-1]
        z = np.concatenate([Hl[a] + Hl[b] + Hl[cc] + Hl[d], Hl[a] * Hl[b] + Hl[cc] * Hl[d],
                            Hl[a] * Hl[pp] + Hl[b] * Hl[qq]], axis=1)
        o = np.maximum(self.mm(z, W["wr1"]) + W["br1"], 0)
        y = o @ W["wr2"] + W["br2"][0]
        c.update(z=z, o=o, idx=(a, b, cc, d, pp, qq), W=W)
        return y, c

    def loss_grad(self, p, swaps, t, mask=None):
        y, c = self.forward(p, swaps)
        m = np.ones(len(y)) if mask is None else (np.asarray(mask) != 0).astype(np.float64)
        cnt = max(m.sum(), 1)
        e = (y - t) * m
        loss = float((e * e).sum() / cnt)
        dy = 2 * e / cnt
        W = c["W"]
        g = {k: np.zeros_like(v) for k, v in W.items()}
        o, z = c["o"], c["z"]
        g["wr2"] = o.T @ dy
        g["br2"] = np.array([dy.sum()])
        do = np.outer(dy, W["wr2"]) * (o > 0)
        g["br1"] = do.sum(0)
        g["wr1"] = self.mm(z.T, do)
        dz = self.mm(do, W["wr1"].T)
        a, b, cc, d, pp, qq = c["idx"]
        Hl = c["H"][-1]
        g0, g1, g2 = dz[:, :H], dz[:, H:2 * H], dz[:, 2 * H:]
        dH = np.zeros_like(Hl)
        np.add.at(dH, a, g0 + g1 * Hl[b] + g2 * Hl[pp])
        np.add.at(dH, b, g0 + g1 * Hl[a] + g2 * Hl[qq])
        np.add.at(dH, cc, g0 + g1 * Hl[d])
        np.add.at(dH, d, g0 + g1 * Hl[cc])
        np.add.at(dH, pp, g2 * Hl[a])
        np.add.at(dH, qq, g2 * Hl[b])
        for l in reversed(range(LAYERS)):
            dpre = dH * (c["H"][l + 1] > 0)
            g[f"b{l}"] = dpre.sum(0)
            g[f"ws{l}"] = self.mm(c["H"][l].T, dpre)
            g[f"wn{l}"] = self.mm(c["M"][l].T, dpre)
            gn = self.mm(dpre, W[f"wn{l}"].T)
            dH = self.mm(dpre, W[f"ws{l}"].T) + self.nbr_mean(gn)  # symmetric adjacency
        dpre = dH * (c["H"][0] > 0)
        g["bin"] = dpre.sum(0)
        g["win"] = self.mm(self.X.T, dpre)
        return loss, pack(g, self.F), y
