"""Inputs of the golden fixtures: seeded graphs written by the library's
generators, and small hand-written files exercising the reader quirks of
graph_t::from_edges (nucleus/graph/graph.hpp:285-411): leading '#'/'%'
comments, the first non-comment line of a bare edge list consumed as a header,
self-loops, duplicates and reversed duplicates, a weight column, 2- and
3-token .mtx headers with 1-based ids, and a .grh round trip."""
import os

import numpy as np

CASES = [
    {"name": "c1_rmat12_ef16_s1", "kind": "rmat", "scale": 12, "ef": 16, "seed": 1, "ext": ".edges"},
    {"name": "rmat10_ef8_s7", "kind": "rmat", "scale": 10, "ef": 8, "seed": 7, "ext": ".edges"},
    {"name": "rmat14_ef16_s4", "kind": "rmat", "scale": 14, "ef": 16, "seed": 4, "ext": ".edges"},
    {"name": "ws2000_k10_s11", "kind": "ws", "n": 2000, "k": 10, "beta": 0.1, "seed": 11, "ext": ".edges"},
    {"name": "rgg20000_d24_s3", "kind": "rgg", "n": 20000, "deg": 24.0, "seed": 3, "ext": ".edges"},
    {"name": "rmat9_ef12_s5_grh", "kind": "rmat", "scale": 9, "ef": 12, "seed": 5, "ext": ".grh"},
    {"name": "quirks_txt", "kind": "text", "ext": ".txt"},
    {"name": "quirks_mtx3", "kind": "mtx3", "ext": ".mtx"},
    {"name": "quirks_mtx2", "kind": "mtx2", "ext": ".mtx"},
    {"name": "rmat13_ef24_s99", "kind": "rmat", "scale": 13, "ef": 24, "seed": 99, "ext": ".edges"},
    {"name": "ws5000_k16_b03_s21", "kind": "ws", "n": 5000, "k": 16, "beta": 0.3, "seed": 21, "ext": ".edges"},
    {"name": "rgg40000_d40_s8", "kind": "rgg", "n": 40000, "deg": 40.0, "seed": 8, "ext": ".edges"},
    {"name": "hubs3000_s2", "kind": "hubs", "n": 3000, "seed": 2, "ext": ".edges"},
    {"name": "cliques4to14", "kind": "cliques", "seed": 5, "ext": ".txt"},
    {"name": "k8_chain40_s6", "kind": "chain", "links": 40, "seed": 6, "ext": ".edges"},
    {"name": "dense300_p05_s12", "kind": "dense", "n": 300, "p": 0.5, "seed": 12, "ext": ".edges"},
]

QUIRKS_TXT = """# a comment line
% another comment
5 6
0 1
0 2
1 2
0 3
1 3
2 3
3 3
0 4
1 4
2 4
3 4
4 0
1 0
2 7\t9
7 8
8 2
7 9
"""

QUIRKS_MTX3 = """%%MatrixMarket matrix coordinate pattern symmetric
% K5 plus a pendant triangle, 1-based ids as written
9 9 14
1 2
1 3
1 4
1 5
2 3
2 4
2 5
3 4
3 5
4 5
5 6
6 7
5 7
7 7
"""

QUIRKS_MTX2 = """%%MatrixMarket
6 12
1 2
1 3
2 3
1 4
2 4
3 4
4 5
5 6
4 6
1 6
2 6
3 6
"""


def structured_pairs(case):
    """Seeded structured graphs (undirected pairs, possibly repeated):
    hubs: three hubs joined to every vertex, a dense 150-vertex core and
      sparse random edges (long, skewed incidence lists);
    cliques: disjoint K4..K14 joined by single bridge edges (k = n - 3 inside
      each clique);
    chain: K8s in a row, each sharing three vertices (a triangle) with the
      next, plus a few random chords;
    dense: G(n, p), every pair independently (long incidence lists on every
      edge and a deep peel)."""
    rng = np.random.default_rng(case["seed"])
    kind = case["kind"]
    pairs = []
    if kind == "hubs":
        n = case["n"]
        for h in range(3):
            pairs += [(h, v) for v in range(3, n)]
        core = np.arange(3, 153)
        for i in range(len(core)):
            for j in range(i + 1, len(core)):
                if rng.random() < 0.3:
                    pairs.append((int(core[i]), int(core[j])))
        a = rng.integers(3, n, 6 * n)
        b = rng.integers(3, n, 6 * n)
        pairs += list(zip(a.tolist(), b.tolist()))
    elif kind == "cliques":
        base = 0
        prev = None
        for size in range(4, 15):
            vs = list(range(base, base + size))
            pairs += [(u, v) for i, u in enumerate(vs) for v in vs[i + 1:]]
            if prev is not None:
                pairs.append((prev, vs[int(rng.integers(0, size))]))
            prev = vs[-1]
            base += size
    elif kind == "dense":
        n = case["n"]
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(len(iu)) < case["p"]
        pairs = list(zip(iu[keep].tolist(), ju[keep].tolist()))
    else:  # chain
        step = 5  # 8 vertices per clique, 3 shared with the next
        for c in range(case["links"]):
            vs = list(range(c * step, c * step + 8))
            pairs += [(u, v) for i, u in enumerate(vs) for v in vs[i + 1:]]
        top = case["links"] * step + 3
        a = rng.integers(0, top, 30)
        b = rng.integers(0, top, 30)
        pairs += list(zip(a.tolist(), b.tolist()))
    perm = rng.permutation(len(pairs))
    src = np.array([pairs[i][0] for i in perm], np.uint32)
    dst = np.array([pairs[i][1] for i in perm], np.uint32)
    return src, dst


def materialise(case, directory):
    """Writes the case's input file into `directory` and returns its path."""
    import nucleus34
    path = os.path.join(directory, case["name"] + case["ext"])
    kind = case["kind"]
    if kind in ("rmat", "ws", "rgg"):
        if kind == "rmat":
            s, d = nucleus34.gen_rmat(case["scale"], case["ef"], case["seed"])
        elif kind == "ws":
            s, d = nucleus34.gen_ws(case["n"], case["k"], case["beta"], case["seed"])
        else:
            s, d = nucleus34.gen_rgg(case["n"], case["deg"], case["seed"])
        if case["ext"] == ".grh":
            nucleus34.save_grh(nucleus34.graph_from_edges(s, d), path)
        else:
            nucleus34.write_edges(s, d, path)
    elif kind in ("hubs", "cliques", "chain", "dense"):
        s, d = structured_pairs(case)
        nucleus34.write_edges(s, d, path)
    else:
        text = {"text": QUIRKS_TXT, "mtx3": QUIRKS_MTX3, "mtx2": QUIRKS_MTX2}[kind]
        with open(path, "w") as f:
            f.write(text)
    return path
