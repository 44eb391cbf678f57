"""The product's Matrix Market reader against the oracle's restatement of
read_mtx (tribit.cu:228-269), including the reference's token-grammar quirks."""
import os

import numpy as np
import pytest

import oracle
from tests.conftest import WIKI_VOTE
import tribit_b200 as tb

HDR = "%%MatrixMarket matrix coordinate pattern general\n"


def both(tmp_path, text, name="g.mtx"):
    p = tmp_path / name
    p.write_bytes(text.encode() if isinstance(text, str) else text)
    st, n, e = oracle.read_mtx(p)
    try:
        n2, e2 = tb.read_mtx(str(p))
        st2 = 0
    except tb.TribitError as ex:
        st2, n2, e2 = ex.status, 0, np.zeros(0, dtype=np.uint64)
    return (st, n, e), (st2, n2, e2)


CASES = {
    "plain": HDR + "% c\n4 4 3\n1 2\n2 3\n3 1\n",
    "values": "%%MatrixMarket matrix coordinate real general\n3 3 3\n1 2 0.5\n2 3 -1e-3\n3 1 7\n",
    "complex_values": "%%MatrixMarket matrix coordinate complex general\n3 3 2\n1 2 1.0 2.0\n2 3 .5 3.\n",
    "selfloops_dups": HDR + "3 3 5\n1 1\n1 2\n2 1\n2 2\n1 3\n",
    "no_trailing_newline": HDR + "3 3 2\n1 2\n2 3",
    "blank_lines": HDR + "3 3 2\n\n1 2\n\n   \n2 3\n",
    "leading_ws": HDR + "3 3 2\n  1 2\n\t2 3\n",
    "trailing_space_eats_next": HDR + "4 4 3\n1 2 \n3 4\n2 3\n",
    "crlf": HDR.replace("\n", "\r\n") + "3 3 2\r\n1 2\r\n2 3\r\n",
    "garbage_stops": HDR + "4 4 3\n1 2\nx y\n3 4\n",
    "comment_in_data_stops": HDR + "4 4 3\n1 2\n% late\n3 4\n",
    "single_token_line": HDR + "4 4 3\n1\n2 3\n4 1\n",
    "symmetric_header": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 2\n",
    "bad_exponent": HDR + "3 3 2\n1 2 1e\n2 3\n",
    "plus_sign_ids": HDR + "3 3 2\n+1 2\n2 +3\n",
    "big_id_overflow_stops": HDR + "3 3 2\n1 2\n4294967297 1\n2 3\n",
    "not_square": HDR + "3 4 1\n1 2\n",
    "no_size_line": HDR + "% only comments\n",
    "empty_entries": HDR + "5 5 0\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_matches_oracle(tmp_path, name):
    (st, n, e), (st2, n2, e2) = both(tmp_path, CASES[name])
    assert st == st2
    if st == 0:
        assert n == n2
        np.testing.assert_array_equal(e, e2)


def test_reader_quirk_semantics(tmp_path):
    (_, _, e), _ = both(tmp_path, CASES["trailing_space_eats_next"])
    # "1 2 \n3 4\n": the value loop swallows "3 4" -> only (0,1) and (1,2) remain
    assert list(e) == [(0 << 32) | 1, (1 << 32) | 2]
    (_, _, e), _ = both(tmp_path, CASES["crlf"])
    assert list(e) == [(0 << 32) | 1]


def test_reader_statuses(tmp_path):
    with pytest.raises(tb.TribitError) as ex:
        tb.read_mtx(str(tmp_path / "missing.mtx"))
    assert ex.value.status == 2
    p = tmp_path / "ns.mtx"
    p.write_text(CASES["not_square"])
    with pytest.raises(tb.TribitError) as ex:
        tb.read_mtx(str(p))
    assert ex.value.status == 4
    p.write_text(CASES["no_size_line"])
    with pytest.raises(tb.TribitError) as ex:
        tb.read_mtx(str(p))
    assert ex.value.status == 3


def test_large_parallel_path_matches(tmp_path):
    e = tb.gen_rmat(17, 16, seed=9)  # ~2M entries, ~25 MB: parallel fast path
    p = tmp_path / "big.mtx"
    tb.write_mtx(str(p), 1 << 17, e)
    assert os.path.getsize(p) > (8 << 20)
    (st, n, a), (st2, n2, b) = both(tmp_path, p.read_bytes(), "big2.mtx")
    assert st == st2 == 0 and n == n2 == 1 << 17
    np.testing.assert_array_equal(a, b)
    # a trailing space on one line forces the exact sequential grammar
    txt = p.read_bytes()
    k = txt.index(b"\n", len(txt) // 2)
    (st, n, a), (st2, n2, b) = both(tmp_path, txt[:k] + b" " + txt[k:], "big3.mtx")
    np.testing.assert_array_equal(a, b)
    assert len(a) == len(e) - 1 - int(np.sum((e >> np.uint64(32)) == (e & np.uint64(0xFFFFFFFF)))) or len(a) < len(e)


def test_large_file_with_mixed_strict_lines_matches(tmp_path):
    # Above the parallel threshold, lines the fast line parser leaves to the
    # per-line strict parse (leading blanks, tabs, value columns, blank lines,
    # self-loops) mixed with plain ones; the last line has no newline.
    rng = np.random.default_rng(3)
    n = 5000
    ids = rng.integers(1, n + 1, size=(900_000, 2))
    forms = ["{} {}", "{}\t{}", "  {} {}", "{}   {} 1.5", "{} {} -2e3", "{} {}"]
    lines = [forms[k].format(a, b) for k, (a, b) in zip(rng.integers(0, len(forms), len(ids)), ids)]
    lines[7] = ""
    lines[100] = "42 42"
    body = "%%MatrixMarket matrix coordinate real general\n% note\n" + f"{n} {n} {len(lines)}\n"
    data = (body + "\n".join(lines)).encode()
    assert len(data) > (8 << 20)
    (st, nn, a), (st2, nn2, b) = both(tmp_path, data, "mixed.mtx")
    assert st == st2 == 0 and nn == nn2 == n
    np.testing.assert_array_equal(a, b)


def test_wiki_vote_reader():
    st, n, a = oracle.read_mtx(WIKI_VOTE)
    n2, b = tb.read_mtx(WIKI_VOTE)
    assert st == 0 and n == n2 == 8297
    np.testing.assert_array_equal(a, b)


def test_write_read_roundtrip(tmp_path):
    e = tb.gen_er(300, 2000, seed=2)
    p = tmp_path / "rt.mtx"
    tb.write_mtx(str(p), 300, e)
    n, back = tb.read_mtx(str(p))
    assert n == 300
    keep = (e >> np.uint64(32)) != (e & np.uint64(0xFFFFFFFF))
    a = e[keep] >> np.uint64(32)
    b = e[keep] & np.uint64(0xFFFFFFFF)
    want = (np.minimum(a, b) << np.uint64(32)) | np.maximum(a, b)
    np.testing.assert_array_equal(back, want)
