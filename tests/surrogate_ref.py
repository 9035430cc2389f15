"""CPU references for the FSC surrogate's kernels (test infrastructure).

The surrogate has no counterpart in the reference project, so its checkers are
restatements of the definitions in include/fos.h:

* ``pairs_and_features``: brute force over all particle pairs, numpy float32
  with the kernels' operation order, so pair sets, normalised distances,
  histograms and features can be compared bit for bit;
* ``mlp_forward_bf16``: the BF16-weight / FP32-accumulate inference in torch;
* ``mlp_loss``: the FP32 training objective in torch autograd.
"""
from __future__ import annotations

import numpy as np
import torch

NB = 11
NF = 16
NH = 64
F = np.float32


def _grid_wrap(p, L):
    """grid.wrapP (grid.py:30-48) in float32: p - L*floor(p*invL + 0.5)."""
    L32, inv = F(L), F(1.0 / L)
    return (p - L32 * np.floor(p * inv + F(0.5))).astype(F)


def owns(i, j):
    """Balanced ownership: pair {a < b} belongs to a when a + b is odd, else to b."""
    return (i < j) == (((i + j) & 1) == 1)


def pairs_and_features(pos, rad, cutoff, L=1.0, chunk=512, nl=None, used=None, fsc=None):
    """All pairs with nd = |d| / (r_i + r_j) < cutoff, each once as (owner i,
    other j), their raw features [P, 16] (include/fos.h order, d = x_j - x_i)
    and the per-particle histograms.  nl [n, 32], used [n] and fsc [n] are the
    last JFA frame's neighbour lists, used counts and fsc (features 14-15;
    zeros when not given)."""
    pos = np.ascontiguousarray(pos, F)
    rad = np.ascontiguousarray(rad, F)
    n = rad.shape[0]
    cut = F(cutoff)
    inv_bins = F(NB) / cut
    hist = np.zeros((n, NB), np.int64)
    I, J, ND = [], [], []
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        d = (pos[None, :, :] - pos[a:b, None, :]).astype(F)
        d = _grid_wrap(d, L)
        d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]).astype(F)
        d2 = (d2 + d[..., 2] * d[..., 2]).astype(F)
        nd = (np.sqrt(d2).astype(F) / (rad[a:b, None] + rad[None, :]).astype(F)).astype(F)
        cand = nd < cut
        cand[np.arange(b - a), np.arange(a, b)] = False
        ii, jj = np.nonzero(cand)
        ii = ii + a
        v = nd[ii - a, jj]
        bins = np.minimum((v * inv_bins).astype(F).astype(np.int64), NB - 1)
        np.add.at(hist, (ii, bins), 1)
        keep = owns(ii, jj)
        I.append(ii[keep])
        J.append(jj[keep])
        ND.append(v[keep])
    I = np.concatenate(I)
    J = np.concatenate(J)
    ND = np.concatenate(ND).astype(F)
    ri, rj = rad[I], rad[J]
    X = np.zeros((len(I), NF), F)
    X[:, 0] = ND
    X[:, 1] = (ri / rj).astype(F)
    den = ((F(2.0) * ND).astype(F) * (ri + rj).astype(F)).astype(F)
    with np.errstate(divide="ignore", invalid="ignore"):
        off = ((ri - rj).astype(F) / den).astype(F)
    X[:, 2] = np.where(ND > 0, off, F(0))
    bins = np.minimum((ND * inv_bins).astype(F).astype(np.int64), NB - 1)
    H = hist[I] + hist[J]
    H[np.arange(len(I)), bins] -= 2
    X[:, 3:3 + NB] = H.astype(F)
    if nl is not None:
        nl = np.asarray(nl)
        u = np.minimum(np.asarray(used), nl.shape[1])
        cols = np.arange(nl.shape[1])[None, :]
        live = cols < u[:, None]
        mem = np.zeros(len(I), bool)
        for a, b in ((I, J), (J, I)):
            mem |= ((nl[a] == b[:, None]) & live[a]).any(axis=1)
        X[:, 3 + NB] = mem.astype(F)
        X[:, 4 + NB] = (np.asarray(fsc)[I] + np.asarray(fsc)[J]).astype(F)
    return {"i": I, "j": J, "nd": ND, "X": X, "hist": hist}


def unpack(params):
    p = torch.as_tensor(np.asarray(params, np.float32))
    o = 0
    W1 = p[o:o + NH * NF].reshape(NH, NF); o += NH * NF
    b1 = p[o:o + NH]; o += NH
    W2 = p[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = p[o:o + NH]; o += NH
    w3 = p[o:o + NH]; o += NH
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def mlp_forward_bf16(X, params, mu, sd):
    """Inference as the kernel computes it: standardise in FP32, round inputs,
    weights and the first hidden layer to BF16, accumulate in FP32 (here FP64
    for a tighter reference)."""
    X = torch.as_tensor(X, dtype=torch.float32).cpu()
    mu = torch.as_tensor(np.asarray(mu, np.float32))
    isd = torch.as_tensor((np.float32(1.0) / np.asarray(sd, np.float32)).astype(np.float32))
    W1, b1, W2, b2, w3, b3 = unpack(params)
    bf = lambda t: t.to(torch.bfloat16).to(torch.float64)
    xs = bf((X - mu) * isd)
    h1 = torch.relu(xs @ bf(W1).T + b1.double())
    h2 = torch.relu(bf(h1) @ bf(W2).T + b2.double())
    z = h2 @ bf(w3) + float(b3)
    return torch.sigmoid(z)


def mlp_loss(X, y, params, mu, sd):
    """FP32 mean BCE-with-logits; returns (loss, params tensor with grad)."""
    X = torch.as_tensor(X, dtype=torch.float32).cpu()
    y = torch.as_tensor(y, dtype=torch.float32).cpu()
    mu = torch.as_tensor(np.asarray(mu, np.float32))
    isd = torch.as_tensor((np.float32(1.0) / np.asarray(sd, np.float32)).astype(np.float32))
    p = torch.tensor(np.asarray(params, np.float32), requires_grad=True)
    o = 0
    W1 = p[o:o + NH * NF].reshape(NH, NF); o += NH * NF
    b1 = p[o:o + NH]; o += NH
    W2 = p[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = p[o:o + NH]; o += NH
    w3 = p[o:o + NH]; o += NH
    b3 = p[o]
    xs = (X - mu) * isd
    h1 = torch.relu(xs @ W1.T + b1)
    h2 = torch.relu(h1 @ W2.T + b2)
    z = h2 @ w3 + b3
    loss = torch.nn.functional.binary_cross_entropy_with_logits(z, y)
    return loss, p
