"""CPU oracle of the learned start vector's network (test infrastructure: only tests/,
the smoke check and the benchmark's checks import it; the product runs the CUDA kernels of
nushellx_b200/csrc/mlp.cu).

A numpy restatement of the same network and the same arithmetic contract:
3 layers n_in -> width -> width -> n_out, SiLU, flat FP32 parameter layout
W1[width][n_in], b1, W2[width][width], b2, W3[n_out][width], b3; hidden activations
rounded to BF16 (round to nearest even) when stored; mean-squared-error loss over
batch x n_out.  With bf16=False and float64 it is the exact network, which the finite-
difference check in tests/ pins.  The reference has no learned component, so this oracle
is pinned by calculus (finite differences), not by reference outputs.
"""
import numpy as np


def bf16_round(x):
    """Round float32 values to the nearest BF16 value (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def layout(n_in, width, n_out):
    shapes = [("W1", (width, n_in)), ("b1", (width,)), ("W2", (width, width)), ("b2", (width,)),
              ("W3", (n_out, width)), ("b3", (n_out,))]
    out, o = {}, 0
    for name, sh in shapes:
        n = int(np.prod(sh))
        out[name] = (o, sh)
        o += n
    return out, o


def unpack(p, n_in, width, n_out):
    lay, n = layout(n_in, width, n_out)
    assert len(p) == n
    return {k: p[o:o + int(np.prod(sh))].reshape(sh) for k, (o, sh) in lay.items()}


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, n_in, width, n_out, bf16=True, dtype=np.float32):
    P = {k: v.astype(dtype) for k, v in unpack(p, n_in, width, n_out).items()}
    x = np.asarray(x, dtype=dtype).reshape(-1, n_in)
    rnd = (lambda a: bf16_round(a).astype(dtype)) if bf16 else (lambda a: a)
    z1 = x @ P["W1"].T + P["b1"]
    a1 = rnd(_silu(z1))
    z2 = a1 @ P["W2"].T + P["b2"]
    a2 = rnd(_silu(z2))
    y = a2 @ P["W3"].T + P["b3"]
    return y, (x, z1, a1, z2, a2)


def loss_and_grad(p, x, t, n_in, width, n_out, bf16=True, dtype=np.float32):
    P = {k: v.astype(dtype) for k, v in unpack(p, n_in, width, n_out).items()}
    y, (x, z1, a1, z2, a2) = forward(p, x, n_in, width, n_out, bf16, dtype)
    t = np.asarray(t, dtype=dtype).reshape(y.shape)
    n = y.size
    d = y - t
    loss = float((d * d).sum() / n)
    dy = (2.0 / n) * d
    g = {"W3": dy.T @ a2, "b3": dy.sum(0)}
    dz2 = (dy @ P["W3"]) * _dsilu(z2)
    g["W2"], g["b2"] = dz2.T @ a1, dz2.sum(0)
    dz1 = (dz2 @ P["W2"]) * _dsilu(z1)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    lay, ntot = layout(n_in, width, n_out)
    flat = np.zeros(ntot, dtype=dtype)
    for k, (o, sh) in lay.items():
        flat[o:o + int(np.prod(sh))] = g[k].ravel()
    return loss, flat
