"""Writes jade_cases.json: the input matrices and expected values of the reference's
jade_complex unit test (src/wannier/jade_complex.hpp, SECTIONs "Even number of
Centers" and "Odd number of Centers"), read from the reference source.

    python tests/golden/make_jade_cases.py <reference root>
"""
import json
import os
import re
import sys


def parse(text):
    cases = []
    for sec in re.split(r'SECTION\("', text)[1:]:
        name = sec.split('"')[0]
        maxsweep = int(re.search(r"int maxsweep = (\d+);", sec).group(1))
        tol = float(re.search(r"double tol = ([0-9.eE+-]+);", sec).group(1))
        a = {}
        for k, i, j, re_, im_ in re.findall(
                r"a\[(\d)\]\[(\d)\]\[(\d)\] = complex\(([-0-9.eE+]+),\s*([-0-9.eE+]+)\);", sec):
            a[f"{k},{i},{j}"] = [float(re_), float(im_)]
        checks = []
        for part, arr, idx, val in re.findall(r"CHECK\((real|imag)\((adiag|u)((?:\[\d\])+)\) == ([-0-9.]+)_a\);", sec):
            checks.append({"part": part, "array": arr, "index": [int(x) for x in re.findall(r"\d", idx)],
                           "value": float(val)})
        n = 1 + max(int(key.split(",")[1]) for key in a)
        cases.append({"name": name, "maxsweep": maxsweep, "tol": tol, "n": n, "a": a, "checks": checks})
    return cases


if __name__ == "__main__":
    ref = sys.argv[1]
    src = open(os.path.join(ref, "src", "wannier", "jade_complex.hpp")).read()
    test = src[src.index("INQ_WANNIER_JADE_COMPLEX_UNIT_TEST"):]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "jade_cases.json")
    json.dump(parse(test), open(out, "w"), indent=1)
    print(out)
