"""FP32 numpy restatement of the scheduler network's forward and backward
passes, with the same BF16 rounding points as the CUDA kernels (weights and
the GEMM operands h1, dh2).  Used by the tests as the CPU reference for the
gradient check."""
from __future__ import annotations

import numpy as np

IN, H, OUT = 781, 256, 4
OFF_W1 = 0
OFF_B1 = OFF_W1 + IN * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * OUT
N_PARAMS = OFF_B3 + OUT


def bf16(x):
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def features(positions):
    """Active input indices per position (list of int arrays)."""
    out = []
    for p in positions:
        bb = [int(p.bb[k]) for k in range(4)]
        occ = bb[1] | bb[2] | bb[3]
        idx = []
        while occ:
            sq = (occ & -occ).bit_length() - 1
            piece = ((bb[1] >> sq) & 1) | (((bb[2] >> sq) & 1) << 1) | (((bb[3] >> sq) & 1) << 2)
            col = (bb[0] >> sq) & 1
            idx.append((col * 6 + piece - 1) * 64 + sq)
            occ &= occ - 1
        if p.color == 0:
            idx.append(768)
        for c in range(4):
            if p.state & (1 << c):
                idx.append(769 + c)
        if p.state >> 4:
            idx.append(773 + (p.state >> 4) - 1)
        out.append(np.array(idx, dtype=np.int64))
    return out


def unpack(params):
    p = np.asarray(params, dtype=np.float32)
    return (p[OFF_W1:OFF_B1].reshape(IN, H), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3].reshape(H, OUT), p[OFF_B3:N_PARAMS])


def forward_backward(params, feats, targets):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    W1b, W2b, W3b = bf16(W1), bf16(W2), bf16(W3)
    n = len(feats)
    h1 = np.stack([b1 + W1b[f].sum(0) for f in feats]).astype(np.float32)
    h1 = np.maximum(h1, 0)
    h1b = bf16(h1)
    h2 = np.maximum(h1b @ W2b + b2, 0)
    y = h2 @ W3b + b3
    t = np.asarray(targets, dtype=np.float32).reshape(n, OUT)
    loss = float(((y - t) ** 2).mean())
    dy = 2 * (y - t) / (n * OUT)
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    dh2 = (dy @ W3b.T) * (h2 > 0)
    gb2 = dh2.sum(0)
    dh2b = bf16(dh2)
    gW2 = h1b.T @ dh2b
    dh1 = (dh2b @ W2b.T) * (h1 > 0)
    gb1 = dh1.sum(0)
    gW1 = np.zeros_like(W1)
    for s, f in enumerate(feats):
        gW1[f] += dh1[s]
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]).astype(np.float32)
    return y, loss, g
