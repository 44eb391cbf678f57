"""Matrix Market ingest on the GPU (tribit_load_mtx) against the host readers.

The GPU parse must yield exactly the entries -- same words, same order -- that
the host reader (tribit_read_mtx) and the oracle's restatement of the
reference's read_mtx (tribit.cu:228-269) give for the same file, across 16 KiB
parse segments and 32 MiB upload pieces, and must hand any file with a line
outside the strict form to the host's exact grammar (load_gpu_parse == 0)."""
import numpy as np
import pytest

import oracle
import tribit_b200 as tb
from tests.conftest import WIKI_VOTE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def counter():
    c = tb.Counter()
    yield c
    c.close()


def check_file(c, path, gpu_parse=True, count_status=0):
    st, n0, want = oracle.read_mtx(str(path))
    assert st == 0
    n1, host = tb.read_mtx(str(path))
    np.testing.assert_array_equal(host, want)
    n, e = c.load_mtx(str(path))
    assert (n, e) == (n0, len(want))
    np.testing.assert_array_equal(c.loaded_entries(), want)
    if count_status:
        # e.g. a '-' id: the grammar wraps it modulo 2^32, past num_nodes
        with pytest.raises(tb.TribitError) as ex:
            c.count_loaded()
        assert ex.value.status == count_status
        return None
    r = c.count_loaded()
    assert r.load_gpu_parse == int(gpu_parse)
    assert (r.triangles, r.edges) == oracle.count(want, n0)
    return r


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode() if isinstance(text, str) else text)
    return p


def test_reference_fixture(counter):
    r = check_file(counter, WIKI_VOTE)
    assert r.triangles == 608389


def test_generated_graph_across_segments_and_pieces(counter, tmp_path):
    # RMAT-20 as text: ~250 MB, eight 32 MiB upload pieces, ~15k parse segments.
    e = tb.gen_rmat(20, 16, seed=20)
    p = tmp_path / "rmat20.mtx"
    tb.write_mtx(str(p), 1 << 20, e)
    assert p.stat().st_size > 200 << 20
    check_file(counter, p)


def test_strict_forms(counter, tmp_path):
    rng = np.random.default_rng(5)
    n = 3000
    ids = rng.integers(1, n + 1, size=(120_000, 2))
    forms = ["{} {}", "{}\t{}", "  {} {}", "{}   {} 1.5", "{} {} -2e3", "{} {} +7 .5 3.", "\t{}\t\t{}\t4E+2"]
    lines = [forms[k].format(a, b) for k, (a, b) in zip(rng.integers(0, len(forms), len(ids)), ids)]
    for k in range(0, len(lines), 997):
        lines[k] = ""  # blank lines
    for k in range(3, len(lines), 1501):
        lines[k] = "   \t "  # blank-only lines
    lines[10] = "42 42"  # self-loop
    body = "%%MatrixMarket matrix coordinate real general\n% c\n%\n" + f"{n} {n} {len(lines)}\n" + "\n".join(lines)
    check_file(counter, write(tmp_path, "forms.mtx", body))  # last line without '\n'
    check_file(counter, write(tmp_path, "forms_nl.mtx", body + "\n"))


def test_long_lines_cross_the_halo(counter, tmp_path):
    # Value tokens longer than a segment's 1 KiB halo, some of them at segment ends.
    rng = np.random.default_rng(6)
    out = ["%%MatrixMarket matrix coordinate real general", "500 500 4000"]
    for k in range(4000):
        a, b = rng.integers(1, 501, size=2)
        tail = " " + "9" * int(rng.integers(1, 3000)) if k % 7 == 0 else ""
        out.append(f"{a} {b}{tail}")
    check_file(counter, write(tmp_path, "long.mtx", "\n".join(out) + "\n"))


def test_empty_and_header_only(counter, tmp_path):
    check_file(counter, write(tmp_path, "empty.mtx", "%%MatrixMarket matrix coordinate pattern general\n5 5 0\n"))
    check_file(counter, write(tmp_path, "noline.mtx", "%%MatrixMarket matrix coordinate pattern general\n5 5 0"))


@pytest.mark.parametrize("name,text,status", [
    ("trailing_blank", "%%MatrixMarket matrix coordinate pattern general\n4 4 3\n1 2 \n2 3\n3 1\n", 0),
    ("crlf", "%%MatrixMarket matrix coordinate pattern general\r\n4 4 3\r\n1 2\r\n2 3\r\n3 1\r\n", 0),
    ("signed_id", "%%MatrixMarket matrix coordinate pattern general\n4 4 3\n1 -2\n2 3\n3 1\n", 5),
    ("plus_id", "%%MatrixMarket matrix coordinate pattern general\n4 4 3\n+1 2\n2 3\n3 1\n", 0),
    ("word_token", "%%MatrixMarket matrix coordinate pattern general\n4 4 4\n1 2\n2 3\nend\n3 1\n", 0),
    ("eleven_digits", "%%MatrixMarket matrix coordinate pattern general\n4 4 2\n1 2\n00000000003 1\n", 0),
])
def test_other_forms_take_the_host_grammar(counter, tmp_path, name, text, status):
    check_file(counter, write(tmp_path, name + ".mtx", text), gpu_parse=False, count_status=status)


def test_errors(counter, tmp_path):
    with pytest.raises(tb.TribitError) as ex:
        counter.load_mtx(str(tmp_path / "missing.mtx"))
    assert ex.value.status == 2
    with pytest.raises(tb.TribitError) as ex:
        counter.load_mtx(str(write(tmp_path, "rect.mtx", "%%MatrixMarket x\n3 4 1\n1 2\n")))
    assert ex.value.status == 4
    # the context stays usable
    check_file(counter, write(tmp_path, "ok.mtx", "%%MatrixMarket x\n3 3 3\n1 2\n2 3\n3 1\n"))


def test_bvgraph_count_matches_oracle(counter, tmp_path):
    # A WebGraph BVGraph (the reference multi-GPU loader's input format,
    # src/multi_gpu/src/main.rs:88), written by the oracle's encoder, counted
    # through tribit_count_bvgraph; its arcs are the oracle's entries.
    from oracle import bvgraph as bv
    from tests.test_bvgraph import structured_graph
    g = structured_graph(6000, 11)
    base = str(tmp_path / "web")
    bv.write(base, g)
    want = oracle.count(bv.entries(g), len(g))
    r = counter.count_bvgraph(base)
    assert (r.triangles, r.edges) == want
