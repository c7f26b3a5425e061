"""The result certificate, checked on the CPU (oracle side).

The device check (nucleus34_ctx_verify) applies three conditions that hold
exactly for the (3,4)-nucleus numbers. Here the oracle's restatement of the
same conditions is shown to accept correct results and to reject planted
mistakes: one triangle's k one too high or one too low, or a death round
moved. The level-synchronous oracle peel that supplies the rounds must give
the bucket peel's k (the numbers are unique)."""
import numpy as np
import pytest

import graphs


def _cases(n34):
    out = []
    for name in sorted(graphs.SMALL):
        s, d = graphs.SMALL[name]()
        out.append((name, n34.graph_from_edges(s, d)))
    a, b = n34.gen_rmat(10, 16, 5)
    out.append(("rmat10", n34.graph_from_edges(a, b)))
    a, b = n34.gen_rgg(3000, 30.0, 6)
    out.append(("rgg3000", n34.graph_from_edges(a, b)))
    a, b = n34.gen_ws(2000, 10, 0.1, 7)
    out.append(("ws2000", n34.graph_from_edges(a, b)))
    return out


def test_certificate_accepts_correct_and_rejects_planted_results(n34, oracle):
    rng = np.random.default_rng(11)
    checked = 0
    for name, g in _cases(n34):
        o = oracle.decompose(g, quds_cap=0)
        if o.T == 0:
            continue
        k, r = oracle.peel_rounds(g, o.tris)
        assert np.array_equal(k, o.k), name
        assert oracle.certify(g, o.tris, k, r) == 0, name
        for t in rng.choice(o.T, size=min(4, o.T), replace=False):
            for dk in (1, -1):
                kb = k.copy()
                kb[t] += dk
                assert oracle.certify(g, o.tris, kb, r) > 0, (name, int(t), dk)
        # a death round moved to another round of a different level
        levels = {int(rr): int(kk) for rr, kk in zip(r, k)}
        t = int(rng.integers(o.T))
        other = [rr for rr, lv in levels.items() if lv != k[t]]
        if other:
            rb = r.copy()
            rb[t] = other[0]
            assert oracle.certify(g, o.tris, k, rb) > 0, name
        checked += 1
    assert checked >= 5
