"""The oracle against its committed golden fixture (tests/golden/oracle_c0_golden.json, written by
tests/golden/make_oracle_golden.py): the stored edit sequence replayed on the depth-10 C0 terrain
gives the same canonical DAG after every edit, the same per-edit counters and the same traced frame.
A change to the oracle that alters any of them fails here; regenerate the fixture only for a change
that is meant to alter results, and say why in the commit."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


@pytest.fixture(scope="module")
def golden(oracle_mod):
    sys.path.insert(0, GOLDEN)
    try:
        import make_oracle_golden as maker
    finally:
        sys.path.remove(GOLDEN)
    with open(os.path.join(GOLDEN, "oracle_c0_golden.json")) as f:
        return maker, json.load(f)


def test_fixture_inputs_are_the_generators(golden):
    maker, fx = golden
    assert fx["levels"] == maker.LEVELS and fx["terrain"] == maker.TERRAIN
    assert [list(v) if isinstance(v, (list, tuple)) else v for v in fx["camera"]] == \
        [list(v) if isinstance(v, (list, tuple)) else v for v in maker.CAMERA]
    assert fx["edit_list"] == maker.edit_list()


def test_oracle_reproduces_the_golden_results(golden):
    maker, fx = golden
    got = maker.run(fx["edit_list"])
    assert got["scene"] == fx["scene"]
    assert len(got["edits"]) == len(fx["edits"]) == 38
    for i, (a, b) in enumerate(zip(got["edits"], fx["edits"])):
        assert a == b, (i, fx["edit_list"][i])
    assert got["frame_sha256"] == fx["frame_sha256"]
    # the fixture exercises every tool and changes the DAG
    assert {d["tool"] for d in fx["edit_list"]} == set(range(9))
    assert len({e["canon"]["root"] for e in fx["edits"]}) > 30
