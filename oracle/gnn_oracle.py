"""CPU oracle of the learned preconditioner network -- TEST INFRASTRUCTURE ONLY.

Only tests/ may import this module, as the oracle of the CUDA forward,
backward and inference kernels in npb-gpu_b200/csrc/gnn.cu; the product
never calls it.  It has no counterpart in the reference (the north-star
addition "learned preconditioner"), so it restates the network as the
library defines it, in NumPy float64:

Matrix scaling.  A (the generator's matrix) is negative definite; the
network sees the SPD matrix scaled by one constant
    A' = -A,  delta = mean(diag(A')),  Ahat = A' / delta
(a per-row scaling would change the spectrum: for this generator Jacobi
scaling slows CG down, so the network's starting point G = I stays plain CG).

Inputs per row i (X, 4 columns): [ahat_ii, s_i, t_i, deg_i / mean_deg] with
s_i = sum_{j!=i} |ahat_ij|, t_i = sum_{j!=i} ahat_ij, deg_i the count of
stored off-diagonal entries.

Network (width 32, FP32 in the library):
    H0 = relu(X W_in + b_in)
    for l in 1..3:  T = H_{l-1} Wm_l;  U = Aoff T;  H_l = relu(H_{l-1} Ws_l + U + b_l)
where Aoff is Ahat without its diagonal.

Output head, on the lower pattern of Ahat (stored (i, j), j <= i):
    g_ii = softplus(H3_i . w_d + c_d)
    g_ij = ahat_ij * (sum_c w_e[c] H3_i[c] H3_j[c] + c_e)     (j < i)
G is lower triangular with a positive diagonal, so M = G^T G is SPD.  The
preconditioner of A' is G^T G / delta, i.e. F = G / sqrt(delta).

Loss over K probe vectors r_k (columns of R):
    L = (1/K) sum_k || Ahat G^T G r_k - r_k ||^2 / ||r_k||^2
Backward uses Ahat (and Aoff) in place of their transposes: A is symmetric
to rounding (the generator forms (j,k) and (k,j) as differently ordered
products), and the CUDA kernels make the same choice.

Parameter vector order (flat, the library's): W_in (4x32, row-major), b_in
(32), then for l = 1..3: Ws_l (32x32), Wm_l (32x32), b_l (32), then w_d (32),
c_d, w_e (32), c_e.
"""
import numpy as np
import scipy.sparse as sp

H = 32
F_IN = 4
N_LAYERS = 3


def param_layout():
    """[(name, shape)] in the flat order the library uses."""
    out = [("W_in", (F_IN, H)), ("b_in", (H,))]
    for l in range(1, N_LAYERS + 1):
        out += [(f"Ws{l}", (H, H)), (f"Wm{l}", (H, H)), (f"b{l}", (H,))]
    out += [("w_d", (H,)), ("c_d", ()), ("w_e", (H,)), ("c_e", ())]
    return out


def n_params():
    return sum(int(np.prod(s)) if s else 1 for _, s in param_layout())


def unflatten(flat):
    flat = np.asarray(flat, np.float64)
    out, k = {}, 0
    for name, shape in param_layout():
        size = int(np.prod(shape)) if shape else 1
        out[name] = flat[k:k + size].reshape(shape) if shape else float(flat[k])
        k += size
    return out


def flatten(p):
    parts = []
    for name, shape in param_layout():
        parts.append(np.atleast_1d(np.asarray(p[name], np.float64)).ravel())
    return np.concatenate(parts)


class Graph:
    """Scaled matrix and its patterns (float64)."""

    def __init__(self, rowstr, colidx, a):
        n = len(rowstr) - 1
        A = sp.csr_matrix((np.asarray(a, np.float64), colidx, rowstr), shape=(n, n))
        Ap = -A
        d = Ap.diagonal()
        if np.any(d <= 0):
            raise ValueError("diag(-A) must be positive")
        delta = float(np.mean(d))
        self.n = n
        self.delta = delta
        self.dscale = np.full(n, 1.0 / np.sqrt(delta))
        self.Ahat = sp.csr_matrix(Ap / delta)
        self.Ahat.sort_indices()
        self.adiag = self.Ahat.diagonal()
        self.Aoff = self.Ahat - sp.diags(self.adiag)
        self.Aoff.eliminate_zeros()
        low = sp.tril(self.Ahat, k=-1).tocsr()
        low.sort_indices()
        self.low = low  # strictly lower part, values ahat_ij
        offdeg = np.diff(self.Aoff.indptr).astype(np.float64)
        mean_deg = max(offdeg.mean(), 1.0)
        absA = abs(self.Aoff)
        self.X = np.stack([self.adiag, np.asarray(absA.sum(axis=1)).ravel(),
                           np.asarray(self.Aoff.sum(axis=1)).ravel(), offdeg / mean_deg], axis=1)


def softplus(u):
    return np.logaddexp(0.0, u)


def sigmoid(u):
    return 1.0 / (1.0 + np.exp(-u))


def forward(p, g):
    """Returns (G as CSR lower incl. diagonal, cache)."""
    relu = lambda z: np.maximum(z, 0.0)
    Hs = []
    h = relu(g.X @ p["W_in"] + p["b_in"])
    Hs.append(h)
    for l in range(1, N_LAYERS + 1):
        T = h @ p[f"Wm{l}"]
        U = g.Aoff @ T
        h = relu(h @ p[f"Ws{l}"] + U + p[f"b{l}"])
        Hs.append(h)
    h3 = Hs[-1]
    ud = h3 @ p["w_d"] + p["c_d"]
    gdiag = softplus(ud)
    rows = np.repeat(np.arange(g.n), np.diff(g.low.indptr))
    cols = g.low.indices
    v = np.einsum("ec,c,ec->e", h3[rows], p["w_e"], h3[cols]) + p["c_e"]
    goff = g.low.data * v
    G = sp.csr_matrix((goff, cols, g.low.indptr), shape=(g.n, g.n)) + sp.diags(gdiag)
    G = sp.csr_matrix(G)
    G.sort_indices()
    cache = dict(Hs=Hs, ud=ud, v=v, rows=rows, cols=cols, gdiag=gdiag, goff=goff)
    return G, cache


def loss_and_grad(p, g, R):
    """L and dL/dparams (dict) for probes R (n x K)."""
    G, c = forward(p, g)
    K = R.shape[1]
    rn2 = np.sum(R * R, axis=0)
    T = G @ R
    U = G.T @ T
    W = g.Ahat @ U - R
    L = float(np.sum(np.sum(W * W, axis=0) / rn2) / K)
    GU = (2.0 / K) * (g.Ahat @ W) / rn2        # dL/dU  (Ahat^T taken as Ahat)
    GT = G @ GU                                  # dL/dT
    # dL/dG_ij = sum_k T_ik GU_jk + GT_ik R_jk  on the lower pattern
    rows, cols = c["rows"], c["cols"]
    dGoff = np.einsum("ek,ek->e", T[rows], GU[cols]) + np.einsum("ek,ek->e", GT[rows], R[cols])
    dGdiag = np.einsum("ik,ik->i", T, GU) + np.einsum("ik,ik->i", GT, R)
    grads = {k: np.zeros_like(np.asarray(v, np.float64)) for k, v in p.items()}
    Hs = c["Hs"]
    h3 = Hs[-1]
    # head
    du = dGdiag * sigmoid(c["ud"])
    dh = np.outer(du, p["w_d"])
    grads["w_d"] = h3.T @ du
    grads["c_d"] = float(du.sum())
    dv = dGoff * g.low.data
    grads["w_e"] = np.einsum("e,ec,ec->c", dv, h3[rows], h3[cols])
    grads["c_e"] = float(dv.sum())
    np.add.at(dh, rows, dv[:, None] * p["w_e"] * h3[cols])
    np.add.at(dh, cols, dv[:, None] * p["w_e"] * h3[rows])
    # message-passing layers
    for l in range(N_LAYERS, 0, -1):
        hprev, hcur = Hs[l - 1], Hs[l]
        dz = dh * (hcur > 0)
        grads[f"Ws{l}"] = hprev.T @ dz
        grads[f"b{l}"] = dz.sum(axis=0)
        dT = g.Aoff @ dz                          # Aoff^T taken as Aoff
        grads[f"Wm{l}"] = hprev.T @ dT
        dh = dz @ p[f"Ws{l}"].T + dT @ p[f"Wm{l}"].T
    dz0 = dh * (Hs[0] > 0)
    grads["W_in"] = g.X.T @ dz0
    grads["b_in"] = dz0.sum(axis=0)
    return L, grads, G


def preconditioner_apply(G, dscale, r):
    """z = F^T F r with F = G diag(dscale) (the preconditioner of A' = -A)."""
    y = dscale * r
    return dscale * (G.T @ (G @ y))
