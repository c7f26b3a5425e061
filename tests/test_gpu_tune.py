"""Scheduling settings of the on-demand variant on the GPU: every setting,
pinned or taken from a tune table, gives the oracle's result bit for bit,
in the regular and the memory-lean layout; the autotuner writes a line that
later runs pick up; the direct variant ignores the table."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETTINGS = [
    {"lane_max": 8},
    {"lane_max": 32},
    {"compact_div": 1},
    {"compact_div": "never"},
    {"sort_shift": 1},
    {"sort_shift": "never"},
    {"rounds_per_replay": 1},
    {"rounds_per_replay": 64},
    {"lane_max": 32, "compact_div": "never", "sort_shift": "never", "rounds_per_replay": 3},
]


@pytest.fixture(scope="module")
def rmat(n34, oracle):
    s, t = n34.gen_rmat(12, 16, 1)
    g = n34.graph_from_edges(s, t)
    return g, oracle.decompose(g, quds_cap=0)


def max_out(g):
    return int(np.max(g.D)) if g.n else 0


@pytest.mark.parametrize("lean", [False, True])
@pytest.mark.parametrize("settings", SETTINGS, ids=[str(s) for s in SETTINGS])
def test_pinned_settings_keep_the_result(n34, rmat, settings, lean):
    g, o = rmat
    flags = n34.OPT_LEAN_MEMORY if lean else 0
    with n34.Context(flags=flags) as ctx:
        ctx.upload(g)
        ctx.set_tune(settings)
        r = ctx.run("ondemand")
        assert ctx.last_tune() == dict(
            {"lane_max": 16, "compact_div": 8, "sort_shift": 12, "rounds_per_replay": 16}, **settings)
        k, tris = ctx.copy_k(r["triangle_count"], with_tris=True)
    assert r["triangle_count"] == o.T and r["four_clique_count"] == o.Q
    assert np.array_equal(tris, o.tris)
    assert np.array_equal(k, o.k)


def test_table_line_applies_to_its_class_only(n34, oracle, rmat, tmp_path):
    g, o = rmat
    table = str(tmp_path / "tune.txt")
    n34.tune_store(table, o.T, g.n, g.m, max_out(g), {"lane_max": 32, "rounds_per_replay": 4})
    with n34.Context(tune_table=table) as ctx:
        ctx.upload(g)
        r = ctx.run("ondemand")
        assert ctx.last_tune() == {"lane_max": 32, "compact_div": 8, "sort_shift": 12, "rounds_per_replay": 4}
        assert np.array_equal(ctx.copy_k(r["triangle_count"]), o.k)
        # the direct variant keeps the defaults
        ctx.run("direct")
        assert ctx.last_tune()["lane_max"] == 16
        # a graph of another class: defaults
        s, t = n34.gen_ws(3000, 10, 0.1, 4)
        g2 = n34.graph_from_edges(s, t)
        ctx.upload(g2)
        r2 = ctx.run("ondemand")
        assert ctx.last_tune()["rounds_per_replay"] == 16
        assert np.array_equal(ctx.copy_k(r2["triangle_count"]), oracle.decompose(g2, quds_cap=0).k)


def test_one_shot_call_reads_the_table(n34, rmat, tmp_path):
    g, o = rmat
    table = str(tmp_path / "tune.txt")
    n34.tune_store(table, o.T, g.n, g.m, max_out(g), {"compact_div": "never", "sort_shift": "never"})
    d = n34.decompose(g, variant="ondemand", tune_table=table)
    assert np.array_equal(d.k, o.k)
    with pytest.raises(n34.Nucleus34Error) as e:
        n34.decompose(g, variant="ondemand", tune_table=str(tmp_path / "absent.txt"))
    assert e.value.code == n34.E_IO


def test_autotune_writes_a_line_that_later_runs_use(n34, rmat, tmp_path):
    g, o = rmat
    table = str(tmp_path / "tune.txt")
    with n34.Context() as ctx:
        ctx.upload(g)
        out = ctx.autotune(table)
        assert out["tuned_sec"] > 0 and out["default_sec"] > 0
        assert out["tuned_sec"] <= out["default_sec"]
        got, matched = n34.tune_lookup(table, o.T, g.n, g.m, max_out(g))
        assert matched and got == out["tune"]
        r = ctx.run("ondemand")  # unpinned: the new line applies
        assert ctx.last_tune() == out["tune"]
        assert np.array_equal(ctx.copy_k(r["triangle_count"]), o.k)


def test_out_of_range_settings_are_rejected(n34):
    with n34.Context() as ctx:
        for bad in ({"lane_max": 12}, {"compact_div": 65}, {"rounds_per_replay": 65}):
            with pytest.raises(n34.Nucleus34Error) as e:
                ctx.set_tune(bad)
            assert e.value.code == n34.E_INVALID
