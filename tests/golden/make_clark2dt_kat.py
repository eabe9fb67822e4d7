"""Generates tests/golden/clark2dt_cdf_inverse.json from the reference's own
unit test of the Clark 2Dt inverse CDF.

The reference pins `clark2dt::cdf_inverse(u01, shape_u, tail_p)`
(necsim/impls/no-std/src/cogs/dispersal_sampler/almost_infinite_clark2dt.rs,
`test_cdf_inverse`) with `assert_eq_bits!` against f64 literals: the jump
distance sqrt(shape_u * (pow_fast_one(1 / (1 - u01), 1 / tail_p) - 1)) that
the AlmostInfinite Clark2Dt dispersal draws (:96-107).  This script reads
that test as text and keeps each case's three arguments and its expected
bits; the literals parse like Rust's (correctly rounded decimal).

Run (where the reference sources are present):
    python tests/golden/make_clark2dt_kat.py [path/to/necsim-rust]
"""
import json
import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REL = "necsim/impls/no-std/src/cogs/dispersal_sampler/almost_infinite_clark2dt.rs"

CASE = re.compile(
    r"cdf_inverse::<ReproducibleMathsCore>\(\s*"
    r"ClosedOpenUnitF64::new\(([0-9._eE+-]+)\)\.unwrap\(\),\s*"
    r"PositiveF64::new\(([0-9._eE+-]+)\)\.unwrap\(\),\s*"
    r"PositiveF64::new\(([0-9._eE+-]+)\)\.unwrap\(\)\s*\),\s*"
    r"([0-9._eE+-]+)\s*\)")


def rust_f64(literal):
    return float(literal.replace("_", ""))


def bits(v):
    return struct.unpack("<Q", struct.pack("<d", v))[0]


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NECSIM_REFERENCE", "/root/reference")
    with open(os.path.join(root, REL)) as f:
        src = f.read()
    cases = []
    for m in CASE.finditer(src):
        u01, shape_u, tail_p, expected = (rust_f64(g) for g in m.groups())
        cases.append({"u01": u01, "shape_u": shape_u, "tail_p": tail_p,
                      "expected_bits": "%016x" % bits(expected), "expected": expected})
    if not cases:
        raise SystemExit("no cdf_inverse cases found in " + REL)
    out = {"source": REL + " (test_cdf_inverse)", "cases": cases}
    with open(os.path.join(HERE, "clark2dt_cdf_inverse.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print("%d cases" % len(cases))


if __name__ == "__main__":
    main()
