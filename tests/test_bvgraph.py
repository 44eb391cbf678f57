"""WebGraph BVGraph input (tribit_read_bvgraph) against the oracle's restatement
of the format (oracle/bvgraph.py), on the CPU.

The oracle's encoder writes basename.graph / .offsets / .properties with
references, copy blocks, intervals and residuals under several code choices;
the product's reader must give exactly the reference loader's words for the
same arcs (every arc x -> y, x != y, as (min << 32) | max in node order,
src/multi_gpu/src/main.rs:142-161), with and without the offsets file (the
parallel and the sequential decoder). The code words themselves are pinned to
the format's definition (gamma, delta, zeta_3, unary)."""
import random

import numpy as np
import pytest

import tribit_b200 as tb
from oracle import bvgraph as bv


def structured_graph(n, seed):
    """Successor lists with runs (intervals), lists shared with recent nodes
    (references and copy blocks), far ids and self-loops."""
    rnd = random.Random(seed)
    g = []
    for x in range(n):
        s = set()
        if rnd.random() < 0.8:
            s |= set(rnd.sample(range(n), rnd.randint(0, 25)))
        if rnd.random() < 0.5:
            base = rnd.randint(0, max(0, n - 40))
            s |= set(range(base, base + rnd.randint(0, 15)))
        if x > 0 and rnd.random() < 0.6:
            src = g[x - rnd.randint(1, min(x, 9))]
            s |= {y for y in src if rnd.random() < 0.8}
        if rnd.random() < 0.1:
            s.add(x)  # self-loop: dropped by the loader
        g.append(sorted(s))
    return g


def test_code_words_follow_the_definition():
    for name, table in bv._check_tables().items():
        for x, word in table.items():
            w = bv.BitWriter()
            {"gamma": w.gamma, "delta": w.delta, "unary": w.unary}.get(name, lambda v: w.zeta(v, 3))(x)
            assert "".join(map(str, w.bits)) == word, (name, x)


def test_oracle_round_trip():
    g = structured_graph(400, 1)
    b, _, p = bv.encode(g)
    assert bv.decode(b, p) == g


CONFIGS = [
    {},
    {"window": 3, "maxref": 1, "minint": 2, "zetak": 2},
    {"window": 0, "minint": 0},
    {"codes": {"OUTDEGREES": "DELTA", "BLOCKS": "DELTA", "RESIDUALS": "GAMMA", "INTERVALS": "DELTA"}},
    {"codes": {"REFERENCES": "GAMMA", "RESIDUALS": "DELTA"}, "zetak": 5},
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=[str(i) for i in range(len(CONFIGS))])
@pytest.mark.parametrize("offsets", [True, False], ids=["offsets", "sequential"])
def test_reader_matches_oracle(tmp_path, cfg, offsets):
    g = structured_graph(5000, 7)
    base = str(tmp_path / "g")
    bv.write(base, g, offsets=offsets, **cfg)
    n, e = tb.read_bvgraph(base)
    assert n == len(g)
    np.testing.assert_array_equal(e, bv.entries(g))


def test_empty_and_isolated(tmp_path):
    base = str(tmp_path / "z")
    bv.write(base, [[] for _ in range(10)])
    n, e = tb.read_bvgraph(base)
    assert n == 10 and e.size == 0
    bv.write(base, [])
    n, e = tb.read_bvgraph(base)
    assert n == 0 and e.size == 0


def test_errors(tmp_path):
    with pytest.raises(tb.TribitError) as ex:
        tb.read_bvgraph(str(tmp_path / "missing"))
    assert ex.value.status == 2
    base = str(tmp_path / "g")
    bv.write(base, structured_graph(300, 3))
    # an unsupported code
    text = open(base + ".properties").read().replace("compressionflags=", "compressionflags=RESIDUALS_NIBBLE")
    open(base + ".properties", "w").write(text)
    with pytest.raises(tb.TribitError) as ex:
        tb.read_bvgraph(base)
    assert ex.value.status == 3
    # a stream cut short
    bv.write(base, structured_graph(300, 3))
    data = open(base + ".graph", "rb").read()
    open(base + ".graph", "wb").write(data[: len(data) // 2])
    with pytest.raises(tb.TribitError) as ex:
        tb.read_bvgraph(base)
    assert ex.value.status == 3
