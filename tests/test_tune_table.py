"""Tune tables of the on-demand variant (host code, no GPU): graph classes,
the nearest-line rule, the writer, and the rejection of malformed tables.

A graph's class is size = floor(log2 T) and skew = floor(log2(max out-degree
* n / m)); a run takes the line of its skew class whose size is nearest,
within 2, ties to the earlier line.
"""
import os

import pytest

DEFAULTS = {"lane_max": 16, "compact_div": 8, "sort_shift": 12, "rounds_per_replay": 16}

# n = 100, m = 400 (mean out-degree 4), max out-degree 16 -> skew 2
N, M, MAXOUT = 100, 400, 16


def write(path, text):
    with open(path, "w") as f:
        f.write(text)
    return str(path)


def test_no_matching_line_gives_the_defaults(n34, tmp_path):
    p = write(tmp_path / "t.txt", "# empty table\n\n")
    got, matched = n34.tune_lookup(p, 1000, N, M, MAXOUT)
    assert got == DEFAULTS and not matched


def test_class_boundaries_are_exact(n34, tmp_path):
    # skew: the largest w with m * 2^w <= max_out * n
    p = write(tmp_path / "t.txt", "size=9 skew=2 lane_max=8\nsize=9 skew=1 lane_max=32\n")
    assert n34.tune_lookup(p, 1000, 10, 40, 16)[0]["lane_max"] == 8    # 40 * 4 == 160: skew 2
    assert n34.tune_lookup(p, 1000, 10, 40, 15)[0]["lane_max"] == 32   # 150 < 160: skew 1
    # size: floor(log2 T); 511 -> 8, 512 -> 9, 1023 -> 9
    p2 = write(tmp_path / "u.txt", "size=8 skew=2 lane_max=8\nsize=9 skew=2 lane_max=32\n")
    assert n34.tune_lookup(p2, 511, N, M, MAXOUT)[0]["lane_max"] == 8
    assert n34.tune_lookup(p2, 512, N, M, MAXOUT)[0]["lane_max"] == 32
    assert n34.tune_lookup(p2, 1023, N, M, MAXOUT)[0]["lane_max"] == 32


def test_nearest_size_within_two_and_ties_to_the_earlier_line(n34, tmp_path):
    p = write(tmp_path / "t.txt", "size=8 skew=2 compact_div=4\nsize=10 skew=2 compact_div=16\n")
    got, matched = n34.tune_lookup(p, 1000, N, M, MAXOUT)   # size 9: both 1 away
    assert matched and got["compact_div"] == 4
    got, _ = n34.tune_lookup(p, 4096, N, M, MAXOUT)         # size 12: 2 away from 10
    assert got["compact_div"] == 16
    got, matched = n34.tune_lookup(p, 8192, N, M, MAXOUT)   # size 13: 3 away
    assert not matched and got == DEFAULTS
    got, matched = n34.tune_lookup(p, 1000, N, M, 1024)     # other skew class
    assert not matched


def test_fields_never_and_comments(n34, tmp_path):
    p = write(tmp_path / "t.txt",
              "# header\n"
              "size=9 skew=2 lane_max=32 compact_div=never sort_shift=never rounds_per_replay=8  # tuned\n")
    got, matched = n34.tune_lookup(p, 1000, N, M, MAXOUT)
    assert matched
    assert got == {"lane_max": 32, "compact_div": "never", "sort_shift": "never", "rounds_per_replay": 8}
    # omitted fields keep their defaults
    p2 = write(tmp_path / "u.txt", "size=9 skew=2 sort_shift=14\n")
    assert n34.tune_lookup(p2, 1000, N, M, MAXOUT)[0] == dict(DEFAULTS, sort_shift=14)


def test_empty_graph_class(n34, tmp_path):
    p = write(tmp_path / "t.txt", "size=0 skew=0 lane_max=8\n")
    got, matched = n34.tune_lookup(p, 0, 0, 0, 0)
    assert matched and got["lane_max"] == 8


@pytest.mark.parametrize("line", [
    "size=9 skew=2 lane_max=12",          # not 8, 16 or 32
    "size=9 skew=2 lane_max=0",
    "size=9 skew=2 compact_div=0",
    "size=9 skew=2 compact_div=65",
    "size=9 skew=2 sort_shift=32",
    "size=9 skew=2 rounds_per_replay=65",
    "size=9 skew=2 rounds_per_replay=-1",
    "size=9 skew=2 lane_max=16 lane_max=8",  # given twice
    "size=9 skew=2 speed=fast",              # unknown key
    "size=9 skew=2 lane_max",                # no value
    "skew=2 lane_max=8",                     # no size
    "size=9 lane_max=8",                     # no skew
    "size=nine skew=2",
    "size=9 skew=2 sec=-1",
    "size=9 skew=2 rounds_per_replay=99999999999",
])
def test_malformed_lines_are_rejected_with_their_line_number(n34, tmp_path, line):
    p = write(tmp_path / "t.txt", "# ok\nsize=1 skew=0\n" + line + "\n")
    with pytest.raises(n34.Nucleus34Error) as e:
        n34.tune_lookup(p, 1000, N, M, MAXOUT)
    assert e.value.code == n34.E_INVALID
    assert ":3:" in str(e.value)


def test_missing_table_is_an_io_error(n34, tmp_path):
    with pytest.raises(n34.Nucleus34Error) as e:
        n34.tune_lookup(str(tmp_path / "absent.txt"), 1000, N, M, MAXOUT)
    assert e.value.code == n34.E_IO


def test_store_creates_replaces_and_appends(n34, tmp_path):
    p = str(tmp_path / "t.txt")
    n34.tune_store(p, 1000, N, M, MAXOUT, {"lane_max": 8}, 1.5, 2.0)
    text = open(p).read().splitlines()
    assert text[0].startswith("#") and len(text) == 2
    assert text[1] == ("size=9 skew=2 lane_max=8 compact_div=8 sort_shift=12 rounds_per_replay=16 "
                       "sec=1.5000 default_sec=2.0000")
    # same class: replaced, comment kept; other class: appended
    n34.tune_store(p, 1023, N, M, MAXOUT, {"compact_div": "never"}, 1.0, 2.0)
    n34.tune_store(p, 1 << 20, N, M, MAXOUT, {"rounds_per_replay": 32})
    lines = open(p).read().splitlines()
    assert len(lines) == 3 and lines[0].startswith("#")
    assert n34.tune_lookup(p, 1000, N, M, MAXOUT)[0] == dict(DEFAULTS, compact_div="never")
    assert n34.tune_lookup(p, 1 << 20, N, M, MAXOUT)[0] == dict(DEFAULTS, rounds_per_replay=32)
    assert not [f for f in os.listdir(tmp_path) if ".tmp." in f]


def test_store_leaves_a_malformed_table_alone(n34, tmp_path):
    p = write(tmp_path / "t.txt", "size=9 skew=2 lane_max=12\n")
    with pytest.raises(n34.Nucleus34Error) as e:
        n34.tune_store(p, 1000, N, M, MAXOUT, {"lane_max": 8})
    assert e.value.code == n34.E_INVALID
    assert open(p).read() == "size=9 skew=2 lane_max=12\n"


def test_store_rejects_settings_out_of_range(n34, tmp_path):
    p = str(tmp_path / "t.txt")
    for bad in ({"lane_max": 12}, {"compact_div": 65}, {"sort_shift": 40}, {"rounds_per_replay": 100}):
        with pytest.raises(n34.Nucleus34Error):
            n34.tune_store(p, 1000, N, M, MAXOUT, bad)
    assert not os.path.exists(p)
    with pytest.raises(ValueError):
        n34.Tune.from_dict({"lanes": 8})


def test_tuning_program_prints_usage_without_arguments():
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "gpu-nucleus34_b200", "bin", "cuNucleus34_tune")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
