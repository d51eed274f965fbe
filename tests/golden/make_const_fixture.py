"""Regenerate tests/golden/const_enums.json from the reference's const.f90.

The reference driver builds its enum dictionaries by splitting each line of
src/const.f90 into whitespace tokens and keeping `name = value,&` triples
(playground/runner/fortdriver/core.py:235-319).  This script applies the same
rule to the reference file and writes the dictionaries as JSON; the test
suite compares sph_playground_b200.consts against the JSON.

Usage: python tests/golden/make_const_fixture.py /root/reference/playground/src/const.f90
"""
import json
import os
import sys

PREFIXES = ["ec_", "es_", "ept_", "ett_", "ebc_", "eeq_", "esd_", "edi_", "eqs_",
            "epc_", "eif_", "ests_"]


def parse(path):
    out = {p[:-1]: {} for p in PREFIXES}
    with open(path) as f:
        for line in f:
            tok = line.split()
            if len(tok) != 3:
                continue
            name, val = tok[0], tok[2]
            for p in PREFIXES:
                if not name.startswith(p):
                    continue
                key = name[len(p):]
                if val.endswith(",&"):
                    val = val[:-2]
                elif p in ("ec_", "es_"):
                    continue  # core.py keeps ec_/es_ only with a trailing ",&"
                if p == "es_" and key == "total":
                    continue
                num = float(val) if p in ("eif_", "ests_") else int(val)
                out[p[:-1]][key] = num
    return out


if __name__ == "__main__":
    src = sys.argv[1]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "const_enums.json")
    with open(dst, "w") as f:
        json.dump(parse(src), f, indent=1, sort_keys=True)
    print("wrote", dst)
