"""The library against the committed golden fixtures (needs a GPU).

In the ordered-f32 reduction mode every published field of every case in tests/golden must hash to
the digest the oracle recorded (make_golden.py), and the reports must match: the fixtures check
the CUDA path bit for bit without running the oracle.
"""
import pytest

import golden_cases as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(G.CASES))
def test_the_library_reproduces_the_fixture(name):
    want = G.oracle_digests()[name]
    got = G.run(G.DeviceSide(), name)
    assert got["sizes"] == want["sizes"]
    assert len(got["reports"]) == len(want["reports"])
    for i, (a, b) in enumerate(zip(got["reports"], want["reports"])):
        assert G.same_report(a, b, G.report_keys(name)), (i, a, b)
    bad = [k for k, h in want["fields"].items() if got["fields"][k] != h]
    assert not bad, f"fields whose bits differ from the fixture: {bad}"
