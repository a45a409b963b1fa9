"""CPU (numpy/scipy, float64) reference of the learned two-level preconditioner.

TEST INFRASTRUCTURE: the checker for the CUDA kernels of the learned preconditioner
(frontistr_b200/csrc/h33_gnn.cuh, h33_coarse.cuh).  It has no counterpart in the
reference solver; its own gradients are checked by finite differences in
tests/test_gnn_reference.py.

Coarse space: aggregates of the node graph (the library's aggregate_nodes, through the
C ABI), Ac = P^T A P, the correction P Ac^-1 P^T.

Prolongator, per node i and aggregate b of i's closed neighbourhood N[i]:
  M_i     = diag of the DOF mask (1 where the row of A has an off-diagonal entry)
  T0(i,b) = D_i^-1 sum_{j in N[i], agg(j) = b} A_ij M_j
  P(i,b)  = [b == agg(i)] M_i - diag(omega_i) T0(i,b)

Network (3 message-passing layers, width 32) producing omega:
  x_i   = [1, (|aggregates of N[i]| - 1) / 7, share of neighbours outside agg(i), M_i]
  s_i   = (trace(D_i)/3)^(-1/2);  e_ij = s_i A_ij s_j  (9 features, edge (i,j), j != i)
  h0_i  = W_in x_i
  w^l_ij = tanh(u_l . e_ij + c_l);  m^l_i = sum_j w^l_ij h^{l-1}_j
  h^l_i = tanh(Ws_l h^{l-1}_i + Wm_l m^l_i)
  out_i = W_out h^3_i;  omega_i = sigmoid(out_i)          (3 per node)

Loss on pairs (r, e) with A e = r (e the error of an iterate): the energy of e outside
the coarse space, relative to its energy:
  L = (e^T r - b^T y) / (e^T r),  b = P^T r,  y = Ac^-1 b
  dL/dP = -2 g y^T / (e^T r),  g = r - A P y;   dL/domega_(i,d) = 2 g_(i,d) (T0 y)_(i,d) / (e^T r)
"""
import numpy as np
import scipy.sparse as sp

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
    """Xavier-like init; W_out starts at scale_out (0 -> omega = 1/2 everywhere)."""
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
        self.blocks = blocks[order].reshape(-1, 3, 3)
        self.E = blocks[order] * (self.s[self.rows] * self.s[self.cols])[:, None]
        self.D = D
        self.N = N


class Coarse:
    """Aggregates, DOF mask, network features and T0 of a matrix (agg from the library)."""

    def __init__(self, m, g, agg):
        N = m.N
        self.N, self.agg = N, np.asarray(agg, dtype=np.int64)
        self.nagg = int(self.agg.max()) + 1
        A = m.to_scipy().tocsr()
        self.A = A
        # DOF mask: rows with an off-diagonal entry
        offd = (A - sp.diags(A.diagonal())).tocsr()
        offd.eliminate_zeros()
        self.mask = (np.diff(offd.indptr) > 0).astype(np.float64)
        M = self.mask.reshape(N, 3)
        # closed-neighbourhood aggregates per node, ascending
        nb = [[i] for i in range(N)]
        for i, j in zip(g.rows, g.cols):
            nb[i].append(j)
        self.pat = [sorted(set(self.agg[nb[i]].tolist())) for i in range(N)]
        # T0(i,b) = D_i^-1 sum_{j in N[i], agg(j)=b} A_ij M_j
        self.T0 = [{b: np.zeros((3, 3)) for b in self.pat[i]} for i in range(N)]
        for i in range(N):
            self.T0[i][self.agg[i]] += g.D[i] * M[i][None, :]
        for k, (i, j) in enumerate(zip(g.rows, g.cols)):
            self.T0[i][self.agg[j]] += g.blocks[k] * M[j][None, :]
        for i in range(N):
            Di = np.linalg.inv(g.D[i])
            for b in self.T0[i]:
                self.T0[i][b] = Di @ self.T0[i][b]
        # network features
        nnb = np.bincount(g.rows, minlength=N)
        nout = np.bincount(g.rows, weights=(self.agg[g.rows] != self.agg[g.cols]).astype(float), minlength=N)
        self.x = np.zeros((N, 6))
        self.x[:, 0] = 1.0
        self.x[:, 1] = np.array([len(p) - 1 for p in self.pat]) / 7.0
        self.x[:, 2] = np.where(nnb > 0, nout / np.maximum(nnb, 1), 0.0)
        self.x[:, 3:] = M

    def prolongator(self, omega, which="P"):
        """P (or T0) as a scipy matrix (3N x 3 nagg) for per-DOF weights omega (3N)."""
        N = self.N
        rows, cols, vals = [], [], []
        w = np.asarray(omega, dtype=np.float64).reshape(N, 3)
        M = self.mask.reshape(N, 3)
        for i in range(N):
            for b in self.pat[i]:
                t = self.T0[i][b]
                if which == "T0":
                    blk = t.copy()
                else:
                    blk = (np.diag(M[i]) if b == self.agg[i] else 0.0) - w[i][:, None] * t
                for d in range(3):
                    for c in range(3):
                        if blk[d, c] != 0.0:
                            rows.append(3 * i + d)
                            cols.append(3 * b + c)
                            vals.append(blk[d, c])
        return sp.csr_matrix((vals, (rows, cols)), shape=(3 * N, 3 * self.nagg))

    def loss_and_grad(self, omega, pairs):
        """Mean loss over pairs (r, e) and dL/domega (3N)."""
        P = self.prolongator(omega)
        T0 = self.prolongator(omega, which="T0")
        Ac = (P.T @ self.A @ P).toarray()
        zero = np.diag(Ac) == 0.0  # a zero basis vector (its DOFs all constrained)
        Ac[zero, zero] = 1.0
        Ainv = np.linalg.inv(Ac)
        L, grad = 0.0, np.zeros(3 * self.N)
        for r, e in pairs:
            er = float(e @ r)
            b = P.T @ r
            y = Ainv @ b
            g = r - self.A @ (P @ y)
            L += (er - b @ y) / er
            grad += 2.0 * g * (T0 @ y) / er
        return L / len(pairs), grad / len(pairs)


def forward(theta, g, x):
    """out (N x 3) and the activations for backward."""
    P = unpack(theta)
    N = g.N
    h = x @ P["W_in"].T
    cache = {"x": x, "h": [h], "m": [], "w": []}
    for l in range(LAYERS):
        w = np.tanh(g.E @ P["u%d" % l] + P["c%d" % l][0])
        m = np.zeros((N, WIDTH))
        np.add.at(m, g.rows, w[:, None] * h[g.cols])
        h = np.tanh(h @ P["Ws%d" % l].T + m @ P["Wm%d" % l].T)
        cache["m"].append(m)
        cache["w"].append(w)
        cache["h"].append(h)
    return h @ P["W_out"].T, cache


def omega_of(out):
    return 1.0 / (1.0 + np.exp(-out))


def backward(theta, g, cache, dout):
    """Gradient of a scalar loss with respect to theta, given dL/dout (N x 3)."""
    P = unpack(theta)
    N = g.N
    dout = dout.reshape(N, 3)
    grads = {name: np.zeros(shp) for name, shp in param_shapes()}
    grads["W_out"] = dout.T @ cache["h"][-1]
    dh = dout @ P["W_out"]
    for l in reversed(range(LAYERS)):
        h_prev, h_new = cache["h"][l], cache["h"][l + 1]
        m, w = cache["m"][l], cache["w"][l]
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


def loss_and_theta_grad(theta, g, c, pairs):
    """The whole chain: theta -> omega -> loss, dL/dtheta and omega."""
    out, cache = forward(theta, g, c.x)
    om = omega_of(out).ravel()
    L, dom = c.loss_and_grad(om, pairs)
    dout = dom * om * (1.0 - om)
    return L, backward(theta, g, cache, dout), om
