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
    else:
        text = {"text": QUIRKS_TXT, "mtx3": QUIRKS_MTX3, "mtx2": QUIRKS_MTX2}[kind]
        with open(path, "w") as f:
            f.write(text)
    return path
