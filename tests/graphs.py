"""Small hand-made graphs with known (3,4)-nucleus answers, and the seeded
synthetic workloads used across the tests."""
import itertools

import numpy as np


def clique(n, offset=0):
    e = [(offset + i, offset + j) for i, j in itertools.combinations(range(n), 2)]
    return np.array([a for a, _ in e], np.uint32), np.array([b for _, b in e], np.uint32)


def union(*parts):
    s = np.concatenate([p[0] for p in parts]).astype(np.uint32)
    d = np.concatenate([p[1] for p in parts]).astype(np.uint32)
    return s, d


def two_k5_sharing_triangle():
    # K5 on {0,1,2,3,4} and K5 on {0,1,2,5,6}: they share triangle {0,1,2}
    a = clique(5)
    b_nodes = [0, 1, 2, 5, 6]
    e = [(b_nodes[i], b_nodes[j]) for i, j in itertools.combinations(range(5), 2)]
    b = (np.array([x for x, _ in e], np.uint32), np.array([y for _, y in e], np.uint32))
    return union(a, b)


def triangle_free(n=50):
    # bipartite: no triangles
    s, d = [], []
    for i in range(n):
        for j in range(n, 2 * n):
            if (i * 7 + j) % 3 == 0:
                s.append(i)
                d.append(j)
    return np.array(s, np.uint32), np.array(d, np.uint32)


def clique_free():
    # a triangulated ring (wheel without hub): triangles but no K4
    n = 30
    s, d = [], []
    for i in range(n):
        s += [i, i]
        d += [(i + 1) % n, (i + 2) % n]
    return np.array(s, np.uint32), np.array(d, np.uint32)


SMALL = {
    "K4": lambda: clique(4),
    "K5": lambda: clique(5),
    "K7": lambda: clique(7),
    "K12": lambda: clique(12),
    "two_K5": two_k5_sharing_triangle,
    "triangle_free": triangle_free,
    "clique_free": clique_free,
    "K6_plus_K4": lambda: union(clique(6), clique(4, offset=10)),
}
