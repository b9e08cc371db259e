"""The committed golden fixtures (tests/golden) against the oracle (no GPU).

known_answers.json holds the reference's published numbers that the oracle tests assert;
oracle_digests.json holds the oracle's outputs on seeded cases (make_golden.py), which the GPU
tests use to check the library bit for bit.  Here the oracle must reproduce every digest: a change
of its arithmetic would move the fixtures away from the pins they were recorded under.
"""
import pytest

import golden_cases as G
from oracle import oracle as O


@pytest.fixture(scope="module")
def digests():
    O.build()
    O.set_threads(min(8, O.max_threads()))
    return G.oracle_digests()


def test_every_case_has_a_fixture(digests):
    assert set(digests) == set(G.CASES)


@pytest.mark.parametrize("name", sorted(G.CASES))
def test_the_oracle_reproduces_its_fixture(digests, name):
    want = digests[name]
    got = G.run(G.OracleSide(), name)
    assert got["sizes"] == want["sizes"]
    assert len(got["reports"]) == len(want["reports"])
    for a, b in zip(got["reports"], want["reports"]):
        assert G.same_report(a, b), (a, b)
    for k, h in want["fields"].items():
        assert got["fields"][k] == h, k


def test_the_fixtures_carry_the_published_iteration_counts(digests):
    """The first-step counts recorded in the fixtures are the published ones."""
    ka = G.known_answers()
    mg = ka["s385_multigrid_iterations"]
    assert digests["s385_32_flat_first_step"]["reports"][0]["iterations"] == mg["flat"]["32"]
    assert digests["s385_32_bump_first_step"]["reports"][0]["iterations"] == mg["bump"]["32"]
    assert digests["s385_64_bump_first_step"]["reports"][0]["iterations"] == mg["bump"]["64"]
    s326 = [r for r in ka["s324_cut_bump_linear"]["rows"] if r["nx"] == 32 and r["jacobi"]][0]
    assert digests["s326_cut_bump_32_linear_step"]["reports"][0]["iterations"] == s326["iterations"]
