"""Every device allocation of a decomposition can fail without leaving the
context broken: with NUCLEUS34_FAIL_ALLOC_AT=N the process's Nth allocation
fails once (a host-side fake of an out-of-memory, no device fault). For
every N the failing call returns E_OOM_BUDGET, and the same context then
decomposes the graph again with the oracle's result. One subprocess per N
(the variable is read once per process)."""
import hashlib
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import hashlib, json, sys
sys.path.insert(0, sys.argv[1])
import nucleus34 as n34
variant, flags = sys.argv[2], int(sys.argv[3])
s, t = n34.gen_rmat(10, 16, 1)
g = n34.graph_from_edges(s, t)
out = {}
with n34.Context(flags=flags) as ctx:
    try:
        ctx.upload(g)
        ctx.run(variant)
        out["first"] = "ok"
    except n34.Nucleus34Error as e:
        out["first"] = [e.code, str(e)]
    # the same context again; the one injected failure may fall here instead
    # (N past the first call's allocations): then it is retried once
    for attempt in range(2):
        try:
            ctx.upload(g)
            r = ctx.run(variant)
            break
        except n34.Nucleus34Error as e:
            if attempt or "injected allocation failure" not in str(e):
                raise
            out["second_injected"] = True
    k = ctx.copy_k(r["triangle_count"])
    out.update(T=r["triangle_count"], Q=r["four_clique_count"], k=hashlib.sha256(k.tobytes()).hexdigest())
print(json.dumps(out))
"""


@pytest.mark.parametrize("variant,flags", [("ondemand", 0), ("direct", 0), ("ondemand", 0x4)])
def test_every_allocation_failure_is_clean(n34, oracle, variant, flags):
    s, t = n34.gen_rmat(10, 16, 1)
    want = oracle.decompose(n34.graph_from_edges(s, t), quds_cap=0)
    want_k = hashlib.sha256(want.k.astype("int32").tobytes()).hexdigest()
    pkg = os.path.join(ROOT, "gpu-nucleus34_b200")
    # Some allocations are optional caches (the entry positions, the frontier
    # order arrays): a failure there is absorbed and the call succeeds. The
    # walk ends when N lies past every allocation of the first call (the
    # injected failure then falls in the second call).
    failures = 0
    for n in range(1, 400):
        env = dict(os.environ, NUCLEUS34_FAIL_ALLOC_AT=str(n))
        r = subprocess.run([sys.executable, "-c", SCRIPT, pkg, variant, str(flags)], capture_output=True,
                           text=True, timeout=300, env=env)
        assert r.returncode == 0, r.stderr[-2000:]
        out = json.loads(r.stdout.strip().splitlines()[-1])
        assert (out["T"], out["Q"], out["k"]) == (want.T, want.Q, want_k), (n, out)
        if out.get("second_injected"):
            assert out["first"] == "ok", (n, out)
            break
        if out["first"] == "ok":
            continue
        code, msg = out["first"]
        assert code == n34.E_OOM_BUDGET and "injected allocation failure" in msg, (n, msg)
        failures += 1
    else:
        pytest.fail("a decomposition made 400 allocations or more")
    assert failures >= 10  # upload, listing, incidence, support and peel all allocate
