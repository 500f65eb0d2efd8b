"""Helpers shared by the GPU parity tests."""
import numpy as np

import oracle


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def oracle_for(sys, settings=None):
    st = dict(sys.settings)
    st.update(settings or {})
    return oracle.Oracle(sys, st["kappa"], st["ctofnb"], st["ctonnb"], st["nfft"], st["order"])


def brute_force_pairs(pos, box, radius, excl_ptr, excl_idx):
    """All minimum-image pairs (i<j) closer than radius that are not
    topologically excluded; returns a set of (i, j)."""
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    n = len(pos)
    nc = np.maximum(1, np.floor(box / radius).astype(int))
    frac = (pos / box + 0.5) % 1.0
    cell = np.minimum((frac * nc).astype(int), nc - 1)
    cid = cell[:, 0] + nc[0] * (cell[:, 1] + nc[1] * cell[:, 2])
    order = np.argsort(cid, kind="stable")
    starts = np.searchsorted(cid[order], np.arange(nc.prod() + 1))
    excl = set()
    for i in range(n):
        for k in range(excl_ptr[i], excl_ptr[i + 1]):
            excl.add((i, int(excl_idx[k])))
    out = set()
    rng = [-1, 0, 1]
    for c in range(int(nc.prod())):
        cx, cy, cz = c % nc[0], (c // nc[0]) % nc[1], c // (nc[0] * nc[1])
        ia = order[starts[c]:starts[c + 1]]
        if len(ia) == 0:
            continue
        nb = set()
        for dx in (rng if nc[0] > 2 else range(nc[0])):
            for dy in (rng if nc[1] > 2 else range(nc[1])):
                for dz in (rng if nc[2] > 2 else range(nc[2])):
                    ox = (cx + dx) % nc[0] if nc[0] > 2 else dx
                    oy = (cy + dy) % nc[1] if nc[1] > 2 else dy
                    oz = (cz + dz) % nc[2] if nc[2] > 2 else dz
                    nb.add(ox + nc[0] * (oy + nc[1] * oz))
        ja = np.concatenate([order[starts[o]:starts[o + 1]] for o in nb])
        d = pos[ia][:, None, :] - pos[ja][None, :, :]
        d -= box * np.round(d / box)
        r2 = (d ** 2).sum(-1)
        ii, jj = np.nonzero(r2 < radius * radius)
        for a, b in zip(ia[ii], ja[jj]):
            if a < b and (int(a), int(b)) not in excl:
                out.add((int(a), int(b)))
    return out
