"""TEST INFRASTRUCTURE — CPU restatement of the learned surrogate's network.

The product computes this network with bf16 tensor-core GEMMs and fp32
accumulation (`physics-engine_b200/csrc/surrogate.cu`); this file restates the
same forward pass and its gradients in numpy, rounding to bf16 at the same
points (every GEMM operand: weights and layer inputs), so the two differ only
by fp32 summation order. Only tests use it, as the checker of the GPU
gradients. The surrogate has no counterpart in the reference, so this is not
pinned to reference outputs ("parity unpinned"): it pins the GPU kernels to
the network's definition.

Network (all MLPs: Linear-ReLU-Linear-ReLU-Linear, hidden width 128):
  h0_i      = enc(f_i)                                  f: 8 node features
  per hop l = 1, 2 (destinations: fluid nodes; edges e = (i <- j)):
    z_e     = h_i Wa + h_j Wb + x_e Wc + b1             x_e: 16 edge features
    m_e     = (relu(relu(z_e) W2 + b2)) W3 + b3
    a_i     = sum_{e into i} m_e
    h_l,i   = h_{l-1},i + node_l([h_{l-1},i, a_i / 16])  (fluid nodes only)
  y_i       = dec(h2_i)                                 4 outputs
  loss      = mean over fluid nodes of sum_c (y_ic - t_ic)^2
"""
from __future__ import annotations

import numpy as np

AGG_SCALE = 1.0 / 16.0


ROUND_BF16 = True  # False: exact arithmetic (for finite-difference checks of the gradients)


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    if not ROUND_BF16:
        return np.asarray(x, np.float64)
    x = np.asarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    rounding = ((b >> 16) & 1) + 0x7FFF
    r = ((b + rounding) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def f32(x):
    """The fp32 storage of a gradient tensor between kernels (exact when not rounding)."""
    return np.asarray(x, np.float32) if ROUND_BF16 else np.asarray(x, np.float64)


def gemm(a, b):
    """a times b with both operands rounded to bf16 (as the tensor cores read
    them) and exact (fp64) accumulation."""
    return np.asarray(bf16(a), np.float64) @ np.asarray(bf16(b), np.float64)


def linear(x, W, b):
    return gemm(x, W) + (0.0 if b is None else b)


class Net:
    """Parameters as dicts of float32 arrays W (K x N) and b (N)."""

    def __init__(self, params):
        self.p = params

    def mlp_fwd(self, name, x):
        p = self.p
        z1 = linear(x, p[name + ".0.W"], p[name + ".0.b"])
        h1 = np.maximum(z1, 0.0)
        z2 = linear(h1, p[name + ".1.W"], p[name + ".1.b"])
        h2 = np.maximum(z2, 0.0)
        y = linear(h2, p[name + ".2.W"], p[name + ".2.b"])
        return y, (x, h1, h2)

    @staticmethod
    def lin_bwd(grads, key, x, W, dz):
        """Backward of x W + b for an fp32 gradient dz: dx = dz W^T and
        dW = x^T dz on bf16 operands, db = column sums of dz."""
        grads[key + ".W"] += gemm(x.T, dz)
        if key + ".b" in grads:
            grads[key + ".b"] += np.asarray(dz, np.float64).sum(0)
        return gemm(dz, W.T)

    def mlp_bwd(self, name, cache, dy, grads):
        p = self.p
        x, h1, h2 = cache
        dy = f32(dy)
        dh2 = self.lin_bwd(grads, name + ".2", h2, p[name + ".2.W"], dy)
        dz2 = f32(dh2 * (h2 > 0))
        dh1 = self.lin_bwd(grads, name + ".1", h1, p[name + ".1.W"], dz2)
        dz1 = f32(dh1 * (h1 > 0))
        return self.lin_bwd(grads, name + ".0", x, p[name + ".0.W"], dz1)

    def forward(self, f, xe, dst, src, fluid):
        """f: nodes x 8; xe: edges x 16; dst/src: edge endpoints; fluid: bool mask."""
        p = self.p
        n = f.shape[0]
        h, c_enc = self.mlp_fwd("enc", f)
        caches = []
        for l in (1, 2):
            pre = f"hop{l}"
            P = linear(h, p[pre + ".edge.a.W"], None)
            Q = linear(h, p[pre + ".edge.b.W"], None)
            z1 = P[dst] + Q[src] + linear(xe, p[pre + ".edge.0.W"], p[pre + ".edge.0.b"])
            h1 = np.maximum(z1, 0.0)
            z2 = linear(h1, p[pre + ".edge.1.W"], p[pre + ".edge.1.b"])
            h2 = np.maximum(z2, 0.0)
            m = linear(h2, p[pre + ".edge.2.W"], p[pre + ".edge.2.b"])
            a = np.zeros((n, m.shape[1]))
            np.add.at(a, dst, m)
            xn = np.concatenate([h, a * AGG_SCALE], axis=1)
            u, c_node = self.mlp_fwd(pre + ".node", xn)
            h_new = h + u * fluid[:, None]
            caches.append((h, z1, h1, h2, c_node))
            h = h_new
        y, c_dec = self.mlp_fwd("dec", h)
        return y, (c_enc, caches, c_dec)

    def loss_and_grads(self, f, xe, dst, src, fluid, target):
        p = self.p
        y, (c_enc, caches, c_dec) = self.forward(f, xe, dst, src, fluid)
        nf = max(int(fluid.sum()), 1)
        diff = (y - target) * fluid[:, None]
        loss = float((diff ** 2).sum() / nf)
        grads = {k: np.zeros(v.shape, np.float64) for k, v in p.items()}
        dy = f32(2.0 * diff / nf)
        dh = self.mlp_bwd("dec", c_dec, dy, grads)
        for l in (2, 1):
            pre = f"hop{l}"
            h, z1, h1, h2, c_node = caches[l - 1]
            du = f32(dh * fluid[:, None])
            dxn = self.mlp_bwd(pre + ".node", c_node, du, grads)
            dh_prev = dh + dxn[:, :128]
            da = dxn[:, 128:] * AGG_SCALE
            dm = f32(da[dst])
            dh2 = self.lin_bwd(grads, pre + ".edge.2", h2, p[pre + ".edge.2.W"], dm)
            dz2 = f32(dh2 * (h2 > 0))
            dh1 = self.lin_bwd(grads, pre + ".edge.1", h1, p[pre + ".edge.1.W"], dz2)
            dz1 = f32(dh1 * (z1 > 0))
            grads[pre + ".edge.0.W"] += gemm(xe.T, dz1)
            grads[pre + ".edge.0.b"] += np.asarray(dz1, np.float64).sum(0)
            dP = np.zeros((h.shape[0], 128))
            dQ = np.zeros((h.shape[0], 128))
            np.add.at(dP, dst, dz1)
            np.add.at(dQ, src, dz1)
            dP, dQ = f32(dP), f32(dQ)
            dh_prev = dh_prev + self.lin_bwd(grads, pre + ".edge.a", h, p[pre + ".edge.a.W"], dP)
            dh_prev = dh_prev + self.lin_bwd(grads, pre + ".edge.b", h, p[pre + ".edge.b.W"], dQ)
            dh = dh_prev
        self.mlp_bwd("enc", c_enc, dh, grads)
        return loss, y, grads
