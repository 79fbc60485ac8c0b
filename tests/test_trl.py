"""Trail-file loader (src/graph.rs) of the library against the oracle's."""
import io

import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic


def both(oracle, text):
    try:
        ref = oracle.parse_trl(text)
    except oracle.OracleError as e:
        ref = e
    try:
        g = bt.Graph.parse(text)
        got = (g.points(), g.starts())
    except bt.BtError as e:
        got = e
    return ref, got


CASES = [
    "0 0 0 1 1\n",
    "0 0 0 1 1\n1 2 2 3 3 4 4\n",
    "id 1 1 1 1 2 2\n",                      # consecutive duplicate dropped (graph.rs:55-58)
    "id 1 1 1 1\nid 0 0 1 1\n",              # first edge collapses to one point: dropped
    "a 1 2\nb 3 4 5 6\n",                    # single-point edge dropped
    "x 0 0 (label) 1 1 <tag> 2 2\n",         # tokens starting with ( or < are skipped
    "x  0 0   1 1\n",                        # empty tokens before an x are skipped
    "x 0 0 1 1\r\ny 2 2 3 3\r\n",            # CRLF
    "x 0 0 1 1\ny 2 2 3 3",                  # no final newline
    "\n\nx 0 0 1 1\n\n",                     # empty lines
    "x 1. 2 .5 3\n",                         # Rust f32 grammar accepts 1. and .5
    "x +1e2 -2E-1 3 4\n",
    "x 0 0 -0.0 0 1 1\n",                    # -0.0 == 0.0: duplicate
    "x 1e-45 0 1 1\n",                       # denormal
]

ERRORS = [
    "",                                      # no drawable edges
    "id 1 1 1 1\n",                          # the only edge collapses: no drawable edges
    "x  0  0   1 1\n",                       # the y token is read unconditionally, "" is invalid
    "x 0 0\n",
    "x 0 0 1\n",                             # unexpected end of line (y)
    "x 0 0 1 (y)\n",                         # y token is parsed, not skipped
    "x 0x10 1 2 2\n",                        # hex floats are not Rust floats
    "x inf 0 1 1\n",                         # non-finite
    "x 1e39 0 1 1\n",                        # overflows to inf
    "x nan 0 1 1\n",
    "x 1,5 0 1 1\n",
    "x 0 0 1 1\ty\n",                        # tab is part of a token
    "x 0 0 1 1\r",                           # lone \r stays in the last line
    "x 1e 2 3 4\n",
    "x . 2 3 4\n",
]


@pytest.mark.parametrize("text", CASES)
def test_parse_matches_oracle(lib, oracle, text):
    ref, got = both(oracle, text)
    assert not isinstance(ref, Exception), ref
    assert not isinstance(got, Exception), got
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[1], ref[1])


@pytest.mark.parametrize("text", ERRORS)
def test_parse_errors_match_oracle(lib, oracle, text):
    ref, got = both(oracle, text)
    assert isinstance(ref, Exception) and isinstance(got, Exception), (ref, got)
    assert got.status == 3
    assert str(ref).split("] ")[-1] == got.message


def test_fuzzed_lines_match_oracle(lib, oracle):
    rng = np.random.default_rng(7)
    tokens = ["0", "1", "-2.5", "3e1", "(a)", "<b>", "", "7.25", "1.", ".5", "x", "+4", "0.1"]
    for _ in range(300):
        lines = []
        for _ in range(rng.integers(1, 6)):
            n = rng.integers(0, 9)
            lines.append(" ".join(["id"] + [tokens[i] for i in rng.integers(0, len(tokens), n)]))
        text = "\n".join(lines)
        ref, got = both(oracle, text)
        if isinstance(ref, Exception):
            assert isinstance(got, Exception), text
            assert str(ref).split("] ")[-1] == got.message, text
        else:
            assert not isinstance(got, Exception), (text, got)
            np.testing.assert_array_equal(got[0], ref[0])
            np.testing.assert_array_equal(got[1], ref[1])


def test_synthetic_roundtrip_and_normalization(lib, oracle, tmp_path):
    w = synthetic.small()
    path = tmp_path / "small.trl"
    synthetic.write_trl(path, w.xy, w.starts)
    g = bt.Graph.load(path)
    np.testing.assert_array_equal(g.points(), w.xy)
    np.testing.assert_array_equal(g.starts(), w.starts)
    ref = oracle.parse_trl(path.read_text())
    np.testing.assert_array_equal(g.normalization(), oracle.normalization(ref[2], ref[3]))


def test_load_missing_file(lib, tmp_path):
    with pytest.raises(bt.BtError) as e:
        bt.Graph.load(tmp_path / "missing.trl")
    assert "read" in e.value.message


def test_write_trl_to_stream():
    buf = io.StringIO()
    synthetic.write_trl(buf, np.float32([[0, 0], [1, 1]]), np.uint32([0, 2]))
    assert buf.getvalue() == "0 0 0 1 1\n"
