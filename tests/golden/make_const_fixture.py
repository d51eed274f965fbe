"""Regenerate tests/golden/const_enums.json from the reference's const.f90.

The reference driver builds its enum dictionaries by splitting each line of
src/const.f90 into whitespace tokens and keeping `name = value,&` triples
(playground/runner/fortdriver/core.py:235-319).  This script applies the same
rule to the reference file and writes the dictionaries as JSON; the test
suite compares sph_playground_b200.consts against the JSON.

Usage: python tests/golden/make_const_fixture.py <reference checkout>/playground/src/const.f90
"""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from sph_playground_b200.consts import parse_const_f90 as parse  # noqa: E402


if __name__ == "__main__":
    src = sys.argv[1]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "const_enums.json")
    with open(dst, "w") as f:
        json.dump(parse(src), f, indent=1, sort_keys=True)
    print("wrote", dst)
