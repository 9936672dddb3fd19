"""FP64 restatement of the visibility-gridding (dimensionality reduction, DR)
data term.

TEST INFRASTRUCTURE ONLY (see ``oracle/nufft.py``).

* ``dr_operator`` -- lib/operators/util_load_data_gen_dr_measurement_operator.m:
  109-228 for one channel (one DR block per channel, no preconditioning):
  H = sum over the channel's data sets of tril(G_curr G_curr') with
  G_curr = G' (:176-177, 208), W = diag(H) > 0 (:213), Lambda = diag(H)^-1/2
  on W (:216), the gridded data Lambda .* (G' y)(W) (:180, 219), H restricted
  to W x W (:217) with its diagonal halved (:220-225).
* ``dr_forward`` / ``dr_adjoint`` -- the istril branches of
  lib/operators/HS_forward_operator_G.m:41-45 (Lambda .* (H u + (u' H)'))
  and HS_adjoint_operator_G.m:46-49 (H' w + H w, w = Lambda .* y).
* ``dr_data_term`` -- the same operator as one sparse matrix per channel,
  Gdr = diag(Lambda) (H + H') S_W (n_W x No), so that the oracle's non-DR
  routines (forward / adjoint / dual update / operator norm / solvers) run the
  DR branch of src/update_dual_data_fidelity.m:85-125 unchanged:
  sc(v2 + Lambda .* (H (2Fx - Fx_old)(W) + ...) - y, eps) is
  sc(v2 + Gdr (2 Fx - Fx_old) - y, eps), g2 += Gdr' v2, and
  norm_res = ||Gdr Fx - y||.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .solvers import DataTerm


def dr_operator(G_blocks, No):
    """Returns (H, W, lam): H (n_W x n_W, lower triangle, diagonal halved),
    W (bool, No), lam (n_W)."""
    H = sp.csr_matrix((No, No), dtype=np.complex128)
    for G in G_blocks:
        Gc = sp.csr_matrix(G).conj().T.tocsr()      # G_curr (No x M)
        H = H + sp.tril(Gc @ Gc.conj().T)
    d = H.diagonal().real
    W = d > 0
    lam = 1.0 / np.sqrt(d[W])
    Hw = sp.csr_matrix(H[W][:, W])
    Hw = Hw - 0.5 * sp.diags(Hw.diagonal())
    return sp.csr_matrix(Hw), W, lam


def dr_forward(H, lam, u):
    """Lambda .* (H u + (u' H)') for u = Fx(W)."""
    return lam * (H @ u + (u.conj() @ H).conj())


def dr_adjoint(H, lam, y):
    """H' w + H w with w = Lambda .* y (the (W) entries of g2)."""
    w = lam * y
    return H.conj().T @ w + H @ w


def dr_reduce_data(G_blocks, y_blocks, W, lam):
    """Lambda .* (G' y)(W): the gridded data of one channel."""
    g = sum(G.conj().T @ yb for G, yb in zip(G_blocks, y_blocks))
    return lam * np.asarray(g).ravel()[W]


def dr_matrix(H, W, lam):
    """Gdr = diag(lam) (H + H') S_W, n_W x No."""
    idx = np.flatnonzero(W)
    Hf = (H + H.conj().T).tocoo()
    return sp.csr_matrix((lam[Hf.row] * Hf.data, (Hf.row, idx[Hf.col])), shape=(len(idx), W.size))


def dr_data_term(data: DataTerm, noise=None, rng=None):
    """DR version of a DataTerm: one block per channel, y_dr = Lambda .* (G'y)(W),
    eps from the gridded noise (util_load_data_gen_dr_measurement_operator.m:
    184-201, 225-227: ||Lambda .* (G' n)(W)||).  ``noise``: per channel, per
    block noise vectors; default: unit complex Gaussian draws (:196-199 with
    sigma 1).  Returns (DataTerm, [(H, W, lam)] per channel)."""
    if rng is None:
        rng = np.random.default_rng(0)
    Gs, ys, eps, ops = [], [], [], []
    for l in range(data.L):
        H, W, lam = dr_operator(data.G[l], data.op.No)
        ops.append((H, W, lam))
        Gs.append([dr_matrix(H, W, lam)])
        ys.append([dr_reduce_data(data.G[l], data.y[l], W, lam)])
        if noise is None:
            nl = [(rng.standard_normal(len(yb)) + 1j * rng.standard_normal(len(yb))) / np.sqrt(2)
                  for yb in data.y[l]]
        else:
            nl = noise[l]
        eps.append([float(np.linalg.norm(dr_reduce_data(data.G[l], nl, W, lam)))])
    return DataTerm(data.op, Gs, ys, eps), ops
