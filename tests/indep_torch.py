"""Independent FP64 restatement of the HDNNP energy in torch (test helper).

Written from the mathematical definitions in the reference (G2/G4 sums of
symmetryFunctions.f90:41-152, tanh^3 cutoff :310-327, scaling hdnnps.f90:471-481,
the MLP of neuralNetworks.f90:94-114) with its own brute-force image search;
forces and dE/dh come from autograd, not from hand-written derivatives.  It is
used only to pin the oracle (tests/test_oracle.py).
"""
from __future__ import annotations

import itertools

import numpy as np
import torch


def _images(lat, rc):
    """Lattice translations that can bring any wrapped atom within rc."""
    if lat is None:
        return np.zeros((1, 3), np.int64)
    h = np.asarray(lat)
    # distance between opposite faces along each reciprocal direction
    inv = np.linalg.inv(h)
    spacing = 1.0 / np.linalg.norm(inv, axis=1)
    n = np.ceil(rc / spacing).astype(int) + 1
    return np.array(list(itertools.product(*[range(-k, k + 1) for k in n])), np.int64)


def energy(model_desc, Z, pos, lat=None):
    """model_desc: dict with 'sfs' {z: (nsf, 11) array as orc_model_sfs},
    'nets' {z: [(W(nout,nin), b, act), ...]}, 'scalesf', 'centersf',
    'atomenergy' (119,), 'rc'.  pos: torch (nat,3) float64 (may require grad);
    lat: torch (3,3) float64 columns = lattice vectors, or None."""
    rc = model_desc["rc"]
    nat = pos.shape[0]
    if lat is not None:
        # wrap into the cell (fractional modulo 1); gradients flow through
        # r = h s with s fixed, as the reference wraps before building lists
        s = torch.linalg.solve(lat, pos.T).T
        s = s - torch.floor(s.detach())
        posw = s @ lat.T
        shifts = torch.tensor(_images(lat.detach().numpy(), rc), dtype=torch.float64) @ lat.T
    else:
        posw = pos
        shifts = torch.zeros((1, 3), dtype=torch.float64)
    Zl = [int(z) for z in Z]
    E = torch.zeros((), dtype=torch.float64)
    for i in range(nat):
        # neighbours of i: all (j, shift) with 0 < |d| < rc (the self image
        # without shift is excluded; other self images are included)
        d_all = posw[i][None, None, :] - (posw[None, :, :] + shifts[:, None, :])  # (ns, nat, 3)
        r2 = (d_all.detach() ** 2).sum(-1)
        mask = r2 < rc * rc
        zero = torch.nonzero(torch.all(shifts.detach() == 0, dim=1))[0, 0]
        mask[zero, i] = False
        si, ji = torch.nonzero(mask, as_tuple=True)
        d = d_all[si, ji]  # dij = r_i - r_j(image)
        el = torch.tensor([Zl[j] for j in ji.tolist()])
        r = torch.sqrt((d * d).sum(-1))
        t = torch.tanh(1.0 - r / rc)
        fc = t ** 3
        sf = model_desc["sfs"][Zl[i]]
        G = []
        n = len(r)
        jj, kk = torch.triu_indices(n, n, 1)
        djk = d[kk] - d[jj]  # (r_i - r_k) - (r_i - r_j) = r_j - r_k
        rjk = torch.sqrt((djk * djk).sum(-1))
        inside = rjk < rc
        fcjk = torch.where(inside, torch.tanh(torch.clamp(1.0 - rjk / rc, min=0.0)) ** 3, torch.zeros_like(rjk))
        cos = (d[jj] * d[kk]).sum(-1) / (r[jj] * r[kk])
        for row in sf:
            typ, e1, e2, _, eta, lam, zeta, rs = row[:8]
            if int(typ) == 2:
                m = el == int(e1)
                G.append((torch.exp(-eta * (r[m] - rs) ** 2) * fc[m]).sum())
            else:
                m = ((el[jj] == int(e1)) & (el[kk] == int(e2))) | ((el[jj] == int(e2)) & (el[kk] == int(e1)))
                term = (2.0 ** (1.0 - zeta)) * (1.0 + lam * cos[m]) ** zeta * torch.exp(
                    -eta * (r[jj][m] ** 2 + r[kk][m] ** 2 + rjk[m] ** 2)
                ) * fc[jj][m] * fc[kk][m] * fcjk[m]
                G.append(term.sum())
        G = torch.stack(G)
        if model_desc["centersf"]:
            G = G - torch.tensor(sf[:, 10])
        if model_desc["scalesf"]:
            G = G / torch.tensor(sf[:, 9] - sf[:, 8])
        x = G
        for W, b, act in model_desc["nets"][Zl[i]]:
            x = torch.tensor(W) @ x + torch.tensor(b)
            if act == "t":
                x = torch.tanh(x)
            elif act == "p":
                x = torch.log1p(torch.exp(x))
            elif act == "r":
                x = torch.relu(x)
        E = E + x[0] + model_desc["atomenergy"][Zl[i]]
    return E


def describe(oracle_model):
    """Builds model_desc from the oracle's parsed model (parsing is tested
    separately; this helper re-uses only the parsed numbers)."""
    s, c, ae = oracle_model.flags()
    return {
        "sfs": {z: oracle_model.sfs(z) for z in oracle_model.elements},
        "nets": {z: oracle_model.net(z) for z in oracle_model.elements},
        "scalesf": s,
        "centersf": c,
        "atomenergy": ae,
        "rc": oracle_model.max_rc,
    }


def energy_forces_dEdLat(desc, Z, pos, lat=None):
    p = torch.tensor(np.asarray(pos), dtype=torch.float64, requires_grad=True)
    L = None
    if lat is not None:
        L = torch.tensor(np.asarray(lat), dtype=torch.float64, requires_grad=True)
        # dE/dh at fixed fractional coordinates: express positions through h
        frac = torch.linalg.solve(L.detach(), p.T).T.detach()
        p_eff = frac @ L.T
        # keep the dependence on p as well: p_eff + (p - p.detach())
        p_eff = p_eff + (p - p.detach())
        E = energy(desc, Z, p_eff, L)
    else:
        E = energy(desc, Z, p, None)
    E.backward()
    F = -p.grad.numpy()
    dl = L.grad.numpy() if L is not None else None
    return float(E.detach()), F, dl
