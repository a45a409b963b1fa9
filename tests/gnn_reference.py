"""CPU (numpy, float64) reference of the learned preconditioner's network.

TEST INFRASTRUCTURE: the checker for the CUDA forward/backward kernels of the
learned preconditioner (frontistr_b200/csrc/h33_gnn.cuh).  It has no counterpart
in the reference solver; its own gradients are checked by finite differences in
tests/test_gnn_reference.py.

Network (3 message-passing layers, width 32, no biases so that it is odd in its
input, and scaled so that it is positively homogeneous -- z(c r) = c z(r)):

  per node i: s_i = (trace(D_i)/3)^(-1/2), zs = SSOR(r), gamma = sqrt(mean(zs^2))
  x_i   = [zs_i / gamma, s_i^2 r_i / gamma]                       (6)
  h0_i  = W_in x_i                                                  (32)
  edge (i,j), j != i, of the matrix graph; e_ij = s_i A_ij s_j      (9, row-major)
  w^l_ij = tanh(u_l . e_ij + c_l)                                   (l = 1..3)
  m^l_i = sum_j w^l_ij h^{l-1}_j
  h^l_i = tanh(Ws_l h^{l-1}_i + Wm_l m^l_i)
  z_i   = zs_i + gamma * W_out h^3_i                                 (3)

Loss on (r, e) pairs with A e = r (e the error of an iterate):
  L = (z - e)^T A (z - e) / (e^T r)       (energy norm, relative)
"""
import numpy as np

WIDTH = 32
LAYERS = 3


def param_shapes():
    shapes = [("W_in", (WIDTH, 6))]
    for l in range(LAYERS):
        shapes += [("u%d" % l, (9,)), ("c%d" % l, (1,)), ("Ws%d" % l, (WIDTH, WIDTH)),
                   ("Wm%d" % l, (WIDTH, WIDTH))]
    shapes.append(("W_out", (3, WIDTH)))
    return shapes


def n_params():
    return sum(int(np.prod(s)) for _, s in param_shapes())


def unpack(theta):
    out, k = {}, 0
    for name, shp in param_shapes():
        n = int(np.prod(shp))
        out[name] = theta[k:k + n].reshape(shp)
        k += n
    return out


def init_params(seed=0, scale_out=0.0):
    """Xavier-like init; W_out starts at scale_out (0 -> the network starts as SSOR)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shp in param_shapes():
        if name == "W_out":
            parts.append(rng.standard_normal(shp).ravel() * scale_out)
        elif name.startswith("u"):
            parts.append(rng.standard_normal(shp).ravel() * 0.3)
        elif name.startswith("c"):
            parts.append(np.full(shp, 0.5).ravel())
        else:
            fan_in = shp[1]
            parts.append(rng.standard_normal(shp).ravel() / np.sqrt(fan_in))
    return np.concatenate(parts)


class Graph:
    """Edges of the matrix graph (both directions) with the scaled block features."""

    def __init__(self, m):
        N = m.N
        D = m.D[:9 * N].reshape(N, 3, 3)
        self.s = 1.0 / np.sqrt(np.trace(D, axis1=1, axis2=2) / 3.0)
        rows, cols, blocks = [], [], []
        for index, item, A in ((m.indexL, m.itemL, m.AL), (m.indexU, m.itemU, m.AU)):
            cnt = np.diff(index[:N + 1])
            rows.append(np.repeat(np.arange(N), cnt))
            cols.append(item[:index[N]] - 1)
            blocks.append(A[:9 * index[N]].reshape(-1, 9))
        rows, cols = np.concatenate(rows), np.concatenate(cols)
        blocks = np.concatenate(blocks)
        order = np.lexsort((cols, rows))
        self.rows, self.cols = rows[order], cols[order]
        self.E = blocks[order] * (self.s[self.rows] * self.s[self.cols])[:, None]
        self.N = N


def forward(theta, g, zs, r):
    P = unpack(theta)
    N = g.N
    zs = zs.reshape(N, 3)
    r = r.reshape(N, 3)
    gamma = np.sqrt(np.mean(zs ** 2))
    x = np.concatenate([zs / gamma, (g.s ** 2)[:, None] * r / gamma], axis=1)
    h = x @ P["W_in"].T
    cache = {"x": x, "gamma": gamma, "h": [h], "m": [], "w": [], "pre_w": []}
    for l in range(LAYERS):
        pre_w = g.E @ P["u%d" % l] + P["c%d" % l][0]
        w = np.tanh(pre_w)
        m = np.zeros((N, WIDTH))
        np.add.at(m, g.rows, w[:, None] * h[g.cols])
        h = np.tanh(h @ P["Ws%d" % l].T + m @ P["Wm%d" % l].T)
        cache["m"].append(m)
        cache["w"].append(w)
        cache["pre_w"].append(pre_w)
        cache["h"].append(h)
    z = zs + gamma * (h @ P["W_out"].T)
    return z.ravel(), cache


def backward(theta, g, cache, dz):
    """Gradient of a scalar loss with respect to theta, given dL/dz."""
    P = unpack(theta)
    N = g.N
    dz = dz.reshape(N, 3)
    grads = {name: np.zeros(shp) for name, shp in param_shapes()}
    gamma = cache["gamma"]
    h3 = cache["h"][-1]
    grads["W_out"] = gamma * dz.T @ h3
    dh = gamma * dz @ P["W_out"]
    for l in reversed(range(LAYERS)):
        h_prev, h_new = cache["h"][l], cache["h"][l + 1]
        m, w, pre_w = cache["m"][l], cache["w"][l], cache["pre_w"][l]
        delta = dh * (1.0 - h_new ** 2)
        grads["Ws%d" % l] = delta.T @ h_prev
        grads["Wm%d" % l] = delta.T @ m
        gm = delta @ P["Wm%d" % l]                       # dL/dm_i
        dh_prev = delta @ P["Ws%d" % l]
        np.add.at(dh_prev, g.cols, w[:, None] * gm[g.rows])
        dw = np.sum(gm[g.rows] * h_prev[g.cols], axis=1)  # dL/dw_ij
        dpre = dw * (1.0 - w ** 2)
        grads["u%d" % l] = g.E.T @ dpre
        grads["c%d" % l] = np.array([dpre.sum()])
        dh = dh_prev
    grads["W_in"] = dh.T @ cache["x"]
    return np.concatenate([grads[name].ravel() for name, _ in param_shapes()])


def energy_loss(A, z, e, r):
    """L = (z-e)^T A (z-e) / (e^T r) and dL/dz."""
    d = z - e
    q = A @ d
    den = float(e @ r)
    return float(d @ q) / den, 2.0 * q / den
