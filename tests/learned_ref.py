"""A plain PyTorch fp64 restatement of the learned SDAINV correction (the
f3r_learned_* kernels): features, network, corrected factors and the loss
1/P sum_p ||Z' W'^T r_p - e_p||^2 / ||e_p||^2 with dense factors, so that
autograd gives the reference gradient.  For small systems only (dense n x n)."""
import numpy as np
import torch

IN_OFFS = lambda nx, sxy: (0, -1, 1, -nx, nx, -sxy, sxy)
Z_OFFS = lambda nx, sxy: (0, 1, nx, sxy)
W_OFFS = lambda nx, sxy: (0, -1, -nx, -sxy)
LAYOUT = {"W1": (0, (64, 7)), "b1": (448, (64,)), "W2": (512, (64, 64)), "b2": (4608, (64,)),
          "W3": (4672, (8, 64)), "b3": (5184, (8,))}


def unpack(p):
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in LAYOUT.items()}


def features(csr, nx, ny):
    r, i, v = csr
    n = len(r) - 1
    offs = IN_OFFS(nx, nx * ny)
    f = np.zeros((n, 7))
    for row in range(n):
        for q in range(r[row], r[row + 1]):
            d = i[q] - row
            if d in offs:
                f[row, offs.index(d)] = np.float32(v[q])  # the kernels read fp32 features
    return f


def slots(csr, offs):
    r, i, _ = csr
    s = np.full(len(i), -1)
    for row in range(len(r) - 1):
        for q in range(r[row], r[row + 1]):
            if i[q] - row in offs:
                s[q] = offs.index(i[q] - row)
    return s


def mlp(p, f):
    P = unpack(p)
    h1 = torch.relu(f @ P["W1"].T + P["b1"])
    h2 = torch.relu(h1 @ P["W2"].T + P["b2"])
    return h2 @ P["W3"].T + P["b3"]


def corrected_dense(csr, sl, delta, slot0):
    r, i, v = csr
    n = len(r) - 1
    rows = np.repeat(np.arange(n), np.diff(r))
    vt = torch.tensor(v, dtype=torch.float64)
    has = torch.tensor(sl >= 0)
    d = delta[torch.tensor(rows), torch.tensor(np.maximum(sl, 0) + slot0)]
    vals = torch.where(has, vt * (1 + d), vt)
    M = torch.zeros(n, n, dtype=torch.float64)
    return M.index_put((torch.tensor(rows), torch.tensor(i.astype(np.int64))), vals)


def loss(params, a, nx, ny, z, wt, r, e):
    """(loss, d loss / d params) in fp64; params a numpy float vector"""
    p = torch.tensor(np.asarray(params, np.float64), requires_grad=True)
    f = torch.tensor(features(a, nx, ny))
    delta = mlp(p, f)
    sxy = nx * ny
    Z = corrected_dense(z, slots(z, Z_OFFS(nx, sxy)), delta, 0)
    W = corrected_dense(wt, slots(wt, W_OFFS(nx, sxy)), delta, 4)
    R = torch.tensor(r)
    E = torch.tensor(e)
    Y = (Z @ (W @ R.T)).T
    L = (((Y - E) ** 2).sum(1) / (E ** 2).sum(1)).mean()
    L.backward()
    return L.item(), p.grad.numpy()


def delta(params, a, nx, ny):
    with torch.no_grad():
        return mlp(torch.tensor(np.asarray(params, np.float64)), torch.tensor(features(a, nx, ny))).numpy()
