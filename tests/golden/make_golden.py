"""Writes oracle_digests.json: the oracle's outputs on the seeded cases of golden_cases.py.

Run from the repository root (it builds the oracle first):

    python tests/golden/make_golden.py

The reference publishes no stored vectors (its pins are the known answers in known_answers.json),
so these fixtures are the oracle's own outputs, recorded once the oracle reproduced every known
answer.  They let the library's tests check its fields bit for bit without running the oracle, and
the oracle's tests catch any change of its arithmetic.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, HERE]

import golden_cases as G  # noqa: E402


def main():
    from oracle import oracle as O
    O.build()
    O.set_threads(O.max_threads())
    side = G.OracleSide()
    out = {name: G.run(side, name) for name in G.CASES}
    with open(os.path.join(HERE, "oracle_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    for name, c in out.items():
        print(name, [r["iterations"] for r in c["reports"]])


if __name__ == "__main__":
    main()
