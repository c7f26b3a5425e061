"""The library's text reader (mapped file, chunked parallel parse, bucketed
CSR build) against the oracle's line-by-line reader on generated files with
every quirk the readers handle: leading comment lines, the header line an
edge list loses, blank lines, tabs, carriage returns, extra columns, comment
and junk lines in the body (skipped), numbers beyond 32 bits (skipped),
self-loops and duplicates. Reader semantics: graph.hpp:285-411."""
import numpy as np
import pytest
from hypothesis import given, settings, HealthCheck
from hypothesis import strategies as st

MAXID = 300

pair = st.tuples(st.integers(0, MAXID), st.integers(0, MAXID))
sep = st.sampled_from([" ", "\t", "  ", " \t "])
lead = st.sampled_from(["", "", " ", "\t"])
tail = st.sampled_from(["", "", " 1", "\t0.5", " 7 extra", "\r", " \r"])
junk = st.sampled_from(["", "abc", "1", "7 x", "-1 2", "+3 4", "# 1 2", "% 5 6", "4294967296 1",
                        "1 99999999999999999999", "12abc 3"])


@st.composite
def body_line(draw):
    kind = draw(st.integers(0, 9))
    if kind < 7:
        s, d = draw(pair)
        if kind == 0:
            d = s  # self-loop
        return f"{draw(lead)}{s}{draw(sep)}{d}{draw(tail)}"
    return draw(junk)


@st.composite
def text_file(draw):
    head = draw(st.lists(st.sampled_from(["# comment", "%% MatrixMarket", "#"]), max_size=3))
    body = draw(st.lists(body_line(), max_size=120))
    ext = draw(st.sampled_from([".edges", ".txt", ".mtx"]))
    header = f"{MAXID + 1} {MAXID + 1} {len(body)}" if ext == ".mtx" else draw(
        st.sampled_from(["1 2", "0 0", "5\t6", "", "header"]))
    end = draw(st.sampled_from(["\n", "\r\n"]))
    text = end.join(head + [header] + body)
    if draw(st.booleans()):
        text += end
    return ext, text


def same_graph(a, b):
    return (a.n == b.n and a.m == b.m and np.array_equal(a.O[: a.n + 1], b.O[: b.n + 1])
            and np.array_equal(a.D, b.D) and np.array_equal(a.E, b.E))


@settings(max_examples=300, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(text_file())
def test_reader_matches_the_oracle(n34, oracle, tmp_path, f):
    ext, text = f
    path = tmp_path / ("g" + ext)
    path.write_bytes(text.encode())
    a = n34.load_graph(str(path))
    b = oracle.read_graph(str(path))
    assert same_graph(a, b), text[:400]


@pytest.mark.parametrize("ext", [".edges", ".mtx"])
def test_reader_matches_the_oracle_across_parse_chunks(n34, oracle, tmp_path, ext):
    """Files of several MB are parsed in chunks cut at line ends; every kind of
    line lands on chunk boundaries somewhere in them."""
    rng = np.random.default_rng(11)
    n = 400_000
    s = rng.integers(0, 60_000, n)
    d = np.where(rng.random(n) < 0.05, s, rng.integers(0, 60_000, n))
    seps = np.array([" ", "\t", "  "])[rng.integers(0, 3, n)]
    tails = np.array(["", " 1", "\r", "\t2.5 x"])[rng.integers(0, 4, n)]
    lines = [f"{a}{p}{b}{t}" for a, p, b, t in zip(s.tolist(), seps.tolist(), d.tolist(), tails.tolist())]
    junk = ["", "# c", "x y", "1", "4294967296 3", "% m"]
    for i in rng.integers(0, n, 5000).tolist():
        lines[i] = junk[i % len(junk)]
    header = f"60000 60000 {n}" if ext == ".mtx" else "1 2"
    text = "% lead comment\n" + header + "\n" + "\n".join(lines) + "\n"
    assert len(text) > 4 << 20
    path = tmp_path / ("big" + ext)
    path.write_bytes(text.encode())
    a = n34.load_graph(str(path))
    b = oracle.read_graph(str(path))
    assert a.m > 300_000
    assert same_graph(a, b)
