"""A numpy shard backend for the sharded VFE protocol, for the CPU tests of
gprx_b200.sharded_value_and_gradient (test infrastructure: it plays the part
of the CUDA handle so the orchestration and the exchange over gloo ranks can
be checked without a GPU).

It restates, for an RbfArd kernel, the same decomposition the CUDA shard
phases use (sgpr.cu): exchange 1 carries this shard's B_s = A_s A_sᵀ,
A_s y_s, Σ_c (k_cc − ‖a_c‖²) over the shard's points (RbfArd: k_cc = 1),
Σ y_s² and n_s; exchange 2 carries H_s = G_s A_sᵀ and the
cross-term gradient ⟨L⁻ᵀ G_s, ∂K(Z, X_s)⟩, with
G_s = B⁻¹A_s − (w r_sᵀ + A_s)/σ², r_s = y_s − A_sᵀ w (the VFE adjoint of
src/sgpr/factor/derivatives.rs:102-144, 283-366).
"""

import math

import numpy as np


def _k(a, b, ls):
    """RbfArd k(a_i, b_j) for rows a (p×d), b (q×d)."""
    d2 = (((a[:, None, :] - b[None, :, :]) / ls) ** 2).sum(-1)
    return np.exp(-0.5 * d2)


def _dk(a, b, ls):
    """∂k/∂log ℓ_f for every feature f: array f × p × q."""
    k = _k(a, b, ls)
    return np.stack([k * ((a[:, None, f] - b[None, :, f]) / ls[f]) ** 2 for f in range(a.shape[1])])


class NumpyShard:
    """Points x (n_s×d), y (n_s); inducing z (m×d); θ = [log ℓ_1..d, log σ²]."""

    def __init__(self, x, y, z):
        self.x, self.y, self.z = np.asarray(x, float), np.asarray(y, float), np.asarray(z, float)
        self.m, self.d = self.z.shape

    def shard_sizes(self):
        m = self.m
        return m * m + m + 3, m * m + self.d + 1

    def shard_assemble(self, params, ex1):
        m, d = self.m, self.d
        self.ls = np.exp(np.asarray(params[:d], float))
        self.s2 = math.exp(params[d])
        kmm = _k(self.z, self.z, self.ls)
        self.L = np.linalg.cholesky(kmm)
        self.A = np.linalg.solve(self.L, _k(self.z, self.x, self.ls))
        e = ex1.numpy()
        e[:m * m] = np.tril(self.A @ self.A.T).reshape(-1, order="F")
        e[m * m:m * m + m] = self.A @ self.y
        e[m * m + m] = (1.0 - (self.A ** 2).sum(axis=0)).sum()
        e[m * m + m + 1] = (self.y ** 2).sum()
        e[m * m + m + 2] = self.x.shape[0]

    def shard_nlml(self, ex1, ex2=None):
        m = self.m
        e = ex1.numpy()
        low = e[:m * m].reshape(m, m, order="F")
        B = np.tril(low) + np.tril(low, -1).T + self.s2 * np.eye(m)
        self.B = B
        self.ay = e[m * m:m * m + m].copy()
        self.tsum, self.y2, self.nt = e[m * m + m], e[m * m + m + 1], e[m * m + m + 2]
        LB = np.linalg.cholesky(B)
        self.w = np.linalg.solve(B, self.ay)
        logdet = (self.nt - m) * math.log(self.s2) + 2.0 * np.log(np.diag(LB)).sum()
        quad = (self.y2 - self.ay @ self.w) / self.s2
        trace = self.tsum / (2.0 * self.s2)
        nl = 0.5 * (self.nt * math.log(2 * math.pi) + logdet + quad) + trace
        if ex2 is not None:
            r = self.y - self.A.T @ self.w
            G = np.linalg.solve(self.B, self.A) - (np.outer(self.w, r) + self.A) / self.s2
            H = G @ self.A.T
            wmn = np.linalg.solve(self.L.T, G)
            dk = _dk(self.z, self.x, self.ls)
            e2 = ex2.numpy()
            e2[:m * m] = H.reshape(-1, order="F")
            e2[m * m:m * m + self.d] = [(wmn * dk[f]).sum() for f in range(self.d)]
            e2[m * m + self.d] = 0.0
        return nl

    def shard_gradient(self, ex2):
        m, d = self.m, self.d
        e2 = ex2.numpy()
        H = e2[:m * m].reshape(m, m, order="F")
        Li = np.linalg.inv(self.L)
        half = np.tril(H, -1) + 0.5 * np.diag(np.diag(H))
        M = Li.T @ half.T @ Li
        wmm = -0.5 * (M + M.T)
        dkm = _dk(self.z, self.z, self.ls)
        g = np.zeros(d + 1)
        for f in range(d):
            g[f] = (wmm * dkm[f]).sum() + e2[m * m + f]  # ∂k_ii/∂θ = 0 for RbfArd
        s2 = self.s2
        trb = np.trace(np.linalg.inv(self.B))
        ww = self.w @ self.w
        quad = (self.y2 - self.ay @ self.w) / s2
        trace = self.tsum / (2.0 * s2)
        d_quad = s2 * ww / s2 - quad
        g[d] = 0.5 * ((self.nt - m) + s2 * trb + d_quad) - trace
        return g
