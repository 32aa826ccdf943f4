"""CPU reference of the learned-window surrogate network (TEST INFRASTRUCTURE).

FP64 numpy forward and backward of the 4-64-64-1 GELU (tanh form) MLP whose
CUDA kernels live in soi_fft_b200/csrc/mlp_kernels.cuh, with the same flat
parameter layout W1[64][4] b1[64] W2[64][64] b2[64] W3[64] b3[1].  Used only to
check the device gradients.
"""
import numpy as np

IN, H = 4, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAMS = OFF_B3 + 1
C = np.sqrt(2.0 / np.pi)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def gelu(x):
    t = np.tanh(C * (x + 0.044715 * x ** 3))
    d = 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * C * (1 + 3 * 0.044715 * x * x)
    return 0.5 * x * (1 + t), d


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    z1 = x @ W1.T + b1
    h1, _ = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2, _ = gelu(z2)
    return h2 @ W3 + b3


def loss_and_grad(p, x, y):
    """mean((f(x) - y)^2) and its gradient with respect to the flat parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = x.shape[0]
    z1 = x @ W1.T + b1
    h1, g1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2, g2 = gelu(z2)
    o = h2 @ W3 + b3
    e = o - y
    loss = np.mean(e * e)
    d3 = 2 * e / n
    d2 = np.outer(d3, W3) * g2
    d1 = (d2 @ W2) * g1
    g = np.zeros(NPARAMS)
    g[OFF_W3:OFF_B3] = d3 @ h2
    g[OFF_B3] = d3.sum()
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


class Net:
    """The same network with IN inputs and OUT outputs (the window proposer of
    soi_fft_b200/window_cheb.py: IN = 2, OUT = 32), layout W1[H][IN] b1[H]
    W2[H][H] b2[H] W3[OUT][H] b3[OUT]; loss = mean over samples and outputs."""

    def __init__(self, n_in, n_out, h=H):
        self.i, self.o, self.h = n_in, n_out, h
        self.offs = np.cumsum([0, h * n_in, h, h * h, h, n_out * h, n_out])
        self.nparams = int(self.offs[-1])

    def unpack(self, p):
        p = np.asarray(p, np.float64)
        o = self.offs
        return (p[o[0]:o[1]].reshape(self.h, self.i), p[o[1]:o[2]], p[o[2]:o[3]].reshape(self.h, self.h),
                p[o[3]:o[4]], p[o[4]:o[5]].reshape(self.o, self.h), p[o[5]:o[6]])

    def forward(self, p, x):
        W1, b1, W2, b2, W3, b3 = self.unpack(p)
        h1, _ = gelu(np.asarray(x, np.float64) @ W1.T + b1)
        h2, _ = gelu(h1 @ W2.T + b2)
        return h2 @ W3.T + b3

    def loss_and_grad(self, p, x, y):
        W1, b1, W2, b2, W3, b3 = self.unpack(p)
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        n = x.shape[0]
        z1 = x @ W1.T + b1
        h1, g1 = gelu(z1)
        z2 = h1 @ W2.T + b2
        h2, g2 = gelu(z2)
        e = h2 @ W3.T + b3 - y
        loss = np.mean(e * e)
        d3 = 2 * e / (n * self.o)
        d2 = (d3 @ W3) * g2
        d1 = (d2 @ W2) * g1
        o = self.offs
        g = np.zeros(self.nparams)
        g[o[4]:o[5]] = (d3.T @ h2).ravel()
        g[o[5]:o[6]] = d3.sum(0)
        g[o[2]:o[3]] = (d2.T @ h1).ravel()
        g[o[3]:o[4]] = d2.sum(0)
        g[o[0]:o[1]] = (d1.T @ x).ravel()
        g[o[1]:o[2]] = d1.sum(0)
        return loss, g
