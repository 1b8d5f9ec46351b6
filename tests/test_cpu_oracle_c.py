"""The C restatement of the graph oracle (oracle/graph_c.c) against the Python
oracle and the reference-generated golden fixtures: identical neighbour lists,
degrees and Cuthill-McKee orders (bit-exact), including the edge-case structure
(pairs exactly at, one ulp inside and outside the cutoff, a duplicate and an
isolated atom) and two disconnected components."""
import os

import numpy as np
import pytest

from oracle import graph as og

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["globule2k", "two_components", "near_cutoff", "shuffled1k"])
def test_c_oracle_matches_reference_goldens(name):
    d = np.load(os.path.join(GOLDEN, f"rcm_{name}.npz"))
    deg, rowptr, cols = og.neighbor_lists_c(d["X"], 8.0)
    assert np.array_equal(deg, d["degree"])
    assert np.array_equal(rowptr, d["rowptr"])
    assert np.array_equal(cols, d["cols"])
    order, undo = og.cuthill_mckee_c(rowptr, cols, deg, seed_order=d["seed_order"])
    assert np.array_equal(order, d["order"])
    assert np.array_equal(undo, d["undo"])


def test_c_oracle_matches_python_oracle():
    from inching_b200 import synth
    X = synth.touching_assembly([1500] * 4, seed=9) / 10.0
    ref = og.neighbor_lists(X, 8.0)
    got = og.neighbor_lists_c(X, 8.0)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    o_ref, u_ref = og.cuthill_mckee(ref[1], ref[2], ref[0])
    o, u = og.cuthill_mckee_c(got[1], got[2], got[0])
    assert np.array_equal(o, o_ref) and np.array_equal(u, u_ref)
