"""CPU oracle: track building of PlaneSite's reconstruction (app/planesite/recon.py:14-54).

TEST INFRASTRUCTURE ONLY (imported by tests/; never by the fieldstitch_b200 package).

Global feature index = offset of the photo + feature index; matches are undirected edges. Tracks
are the connected components (scipy.sparse.csgraph, which labels the components of an undirected
graph in the order of their smallest node) of the matched features, without the components that
hold two features of one photo or fewer than two features, renumbered in label order;
observations listed by track, then global index.
"""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components


def build_tracks(pairs, nfeat, n_img):
    off = np.r_[0, np.cumsum(np.asarray(nfeat, np.int64))]
    z = np.zeros(0, np.int64)
    if not pairs:
        return z, z, z, 0
    u = np.concatenate([off[i] + np.asarray(q, np.int64) for i, j, q, t in pairs])
    v = np.concatenate([off[j] + np.asarray(t, np.int64) for i, j, q, t in pairs])
    T = int(off[-1])
    if len(u) == 0 or T == 0:
        return z, z, z, 0
    g = sp.coo_matrix((np.ones(len(u), np.int8), (u, v)), shape=(T, T))
    ncomp, lab = connected_components(g, directed=False)
    nodes = np.unique(np.r_[u, v])
    comp = lab[nodes].astype(np.int64)
    photo = np.searchsorted(off, nodes, side="right") - 1
    # components holding two features of one photo
    pk = comp * n_img + photo
    s = np.sort(pk)
    bad = np.zeros(ncomp, bool)
    bad[s[1:][s[1:] == s[:-1]] // n_img] = True
    size = np.bincount(comp, minlength=ncomp)
    keep = ~bad[comp] & (size[comp] >= 2)
    comp, photo, nodes = comp[keep], photo[keep], nodes[keep]
    live = np.zeros(ncomp, bool)
    live[comp] = True
    tid = (np.cumsum(live) - 1)[comp]
    order = np.lexsort((nodes, tid))
    return tid[order], photo[order], (nodes - off[photo])[order], int(live.sum())
