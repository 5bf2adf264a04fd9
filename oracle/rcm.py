"""Test infrastructure only: a plain-Python restatement of the reverse
Cuthill-McKee cell order that the product's mesh builder computes
(fcfd_mesh_rcm), used by tests/ as the checker of that integer output.

The reference has no locality renumbering (its cell order is the grid file's
element order, or ParMETIS's when partitioned: grid_partition.cc:25-141), so
this is a restatement of the published algorithm the product follows, with
the product's tie rules: Cuthill & McKee (1969) breadth-first order over the
face-neighbour graph of the interior cells, each cell's unvisited neighbours
in ascending (degree, index); per connected component a pseudo-peripheral
start cell found by the George-Liu search (from the least-degree,
lowest-index cell of the component, move to the least-degree cell of the
last breadth-first level while the eccentricity grows); components in the
order of their least-degree, lowest-index cell; the whole sequence reversed
(George 1971).  perm[new] = old.
"""
import numpy as np


def _graph(nc, face_parent, face_neighbor, face_bc):
    nbrs = [set() for _ in range(nc)]
    for p, n, b in zip(face_parent, face_neighbor, face_bc):
        if b >= 0 or p < 0 or n < 0 or p >= nc or n >= nc or p == n:
            continue
        nbrs[p].add(int(n))
        nbrs[n].add(int(p))
    deg = [len(s) for s in nbrs]
    adj = [sorted(s, key=lambda o: (deg[o], o)) for s in nbrs]
    return adj, deg


def _last_level(adj, deg, done, r):
    level = {r: 0}
    cur, last, ecc = [r], [r], 0
    while cur:
        nxt = []
        for c in cur:
            for o in adj[c]:
                if done[o] or o in level:
                    continue
                level[o] = level[c] + 1
                nxt.append(o)
        if not nxt:
            break
        ecc += 1
        last, cur = nxt, nxt
    best = min(last, key=lambda c: (deg[c], c))
    return best, ecc


def rcm_order(nc, face_parent, face_neighbor, face_bc):
    adj, deg = _graph(nc, face_parent, face_neighbor, face_bc)
    done = [False] * nc
    order = []
    while True:
        rest = [c for c in range(nc) if not done[c]]
        if not rest:
            break
        seed = min(rest, key=lambda c: (deg[c], c))
        cand, ecc = _last_level(adj, deg, done, seed)
        while True:
            cand2, ecc2 = _last_level(adj, deg, done, cand)
            if ecc2 <= ecc:
                break
            seed, ecc, cand = cand, ecc2, cand2
        head = len(order)
        order.append(seed)
        done[seed] = True
        while head < len(order):
            c = order[head]
            head += 1
            for o in adj[c]:
                if not done[o]:
                    done[o] = True
                    order.append(o)
    return np.array(order[::-1], dtype=np.int32)
