#!/usr/bin/env python3
"""Generate the committed golden fixtures under tests/golden/.

* ``kats.json``: the closed-form known-answer tests of the reference's own
  test drivers (TALSH/test.cpp, TALSH/main.F90), restated as data, plus
  digital patterns and TTGT permutations derived by hand from the definitions
  in TALSH/tensor_algebra_cpu.F90:5307-5531 (get_contr_pattern_dig) and
  :5613-5755 (get_contr_permutations).  These are written out literally below;
  nothing here is computed by the oracle.
* ``ctm_patterns.json``: the 48 contraction patterns with their tensor shapes
  from TALSH/tensor_contractions.txt, the corpus of the reference's
  ``benchmark_tensor_contractions_ctm`` (TALSH/main.F90:912-1026; format per
  :962-963: a pattern line, then "rank dims... rank dims... rank dims...").
  This part reads the reference tree and is run only where it is mounted.

Usage: python tests/golden/make_golden.py [--reference-root DIR]   (or TALSH_REFERENCE_ROOT=DIR)
"""
import argparse
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))

KATS = {
    "patterns": [
        # pattern, expected (cptrn, drank, lrank, rrank, conj_bits), derivation note
        {"pattern": "D(a,b,c,d)+=L(c,k,a,l)*R(l,d,k,b)", "cptrn": [3, -3, 1, -1, -4, 4, -2, 2],
         "ranks": [4, 4, 4], "conj": 0, "note": "single-block R8 contraction of the 40^4 workload"},
        {"pattern": "D(a,b,c,d)+=L(d,c,k,l)*R(b,a,k,l)", "cptrn": [4, 3, -3, -4, 2, 1, -3, -4],
         "ranks": [4, 4, 4], "conj": 0, "note": "digital pattern written by hand in TALSH/test.cpp:1094"},
        {"pattern": "D(a,b,i,j)+=L(c,b,d,a)*R(j,d,i,c)", "cptrn": [-4, 2, -2, 1, 4, -3, 3, -1],
         "ranks": [4, 4, 4], "conj": 0, "note": "TALSH/test.cpp:120"},
        {"pattern": "D(a,b,c,d)=L(c,d,b,a)", "cptrn": [3, 4, 2, 1], "ranks": [4, 4, -1], "conj": 0,
         "note": "copy pattern of the talsh.h:495 comment"},
        {"pattern": "D(a,b)+=L+(c,a)*R(c,b)", "cptrn": [-1, 1, -1, 2], "ranks": [2, 2, 2], "conj": 2,
         "note": "conjugated left operand (tensor_algebra_cpu.F90:5380)"},
        {"pattern": "D+(a,b)+=L(c,a)*R+(c,b)", "cptrn": [-1, 1, -1, 2], "ranks": [2, 2, 2], "conj": 5,
         "note": "conjugated destination and right operand"},
        {"pattern": "D(a,b)+=L(c+,a)*R(c,b+)", "cptrn": [-1, 1, -1, 2], "ranks": [2, 2, 2], "conj": 0,
         "note": "contravariant '+' suffixes are stripped before matching (:5336-5339)"},
        {"pattern": "D()+=L(a,b)*R(b,a)", "cptrn": [-2, -1, -2, -1], "ranks": [0, 2, 2], "conj": 0,
         "note": "full contraction into a scalar (TALSH/test.cpp:356)"},
        {"pattern": "D(a,b)+=L(c,d)*R(d,a,b,c)", "cptrn": [-4, -1, -2, 1, 2, -1], "ranks": [2, 2, 4],
         "conj": 0, "note": "TALSH/test.cpp:964"},
        {"pattern": "D(a,b,c,d)+=L(p,c,a)*R(p,b,d)", "cptrn": [-1, 3, 1, -1, 2, 4], "ranks": [4, 3, 3],
         "conj": 0, "note": "TALSH/main.F90:392"},
        {"pattern": "D(a,b,c)+=L(b,d,a)*R(d,c)", "cptrn": [2, -1, 1, -2, 3], "ranks": [3, 3, 2],
         "conj": 0, "note": "first entry of TALSH/tensor_contractions.txt"},
        {"pattern": "D(a|b)+=L(c|a)*R(c|b)", "cptrn": [-1, 1, -1, 2], "ranks": [2, 2, 2], "conj": 0,
         "note": "'|' is an index separator like ','"},
        {"pattern": "D(ia1,ib2)+=L(ib2,k2+,c3)*R+(c3+,ia1,k2)", "cptrn": [2, -3, -1, -3, 1, -2],
         "ranks": [2, 3, 3], "conj": 4, "note": "example in the get_contr_pattern_dig header, :5310"},
    ],
    "pattern_errors": [
        # malformed patterns must be rejected (any nonzero code); expected reference code noted
        {"pattern": "", "code": 16},
        {"pattern": "D(a,b)+=L(c,a)*R(c,b,d)", "code": 7, "note": "d appears once, as the last label"},
        {"pattern": "D(a,b,d)+=L(c,a)*R(c,b)", "code": 11, "note": "d appears once"},
        {"pattern": "D(a,a)+=L(c,a)*R(c,a)", "code": 10, "note": "repeated destination index"},
        {"pattern": "D(a,b)+=L(c,a)*R(c,b_)", "code": 4, "note": "'_' is not alphanumeric"},
        {"pattern": "D(a,,b)+=L(c,a)*R(c,b)", "code": 2, "note": "empty label"},
        {"pattern": "D(a,b)+=L(c,a)*R(c,b)*S(a)", "code": 1, "note": "three inputs"},
        {"pattern": "D(a,b)+=L(c,a)*R(c,b", "code": 5, "note": "unclosed parenthesis"},
        {"pattern": "D(a,)+=L(a)", "code": 3, "note": "separator before ')'"},
        {"pattern": "D(a)=L(a,c,c)", "code": 13, "note": "unary with an index repeated in L"},
        {"pattern": "D(a,b)=L(b,c)", "code": 14, "note": "unary with a destination index missing from L"},
    ],
    "permutations": [
        # get_contr_permutations(1,0,...) derived by hand from :5613-5755
        {"cptrn": [3, -3, 1, -1, -4, 4, -2, 2], "lrank": 4, "rrank": 4, "conj": 0,
         "dprm": [3, 1, 4, 2], "lprm": [3, 2, 4, 1], "rprm": [1, 3, 2, 4], "ncd": 2, "nlu": 2, "nru": 2},
        {"cptrn": [4, 3, -3, -4, 2, 1, -3, -4], "lrank": 4, "rrank": 4, "conj": 0,
         "dprm": [4, 3, 2, 1], "lprm": [3, 4, 1, 2], "rprm": [3, 4, 1, 2], "ncd": 2, "nlu": 2, "nru": 2},
        {"cptrn": [-1, 1, 2, -1, 3, 4], "lrank": 3, "rrank": 3, "conj": 0,
         "dprm": [1, 2, 3, 4], "lprm": [1, 2, 3], "rprm": [1, 2, 3], "ncd": 1, "nlu": 2, "nru": 2,
         "note": "D(a,b,c,d)+=L(k,a,b)*R(k,c,d): already matricized, the 'simple' rule keeps D"},
        {"cptrn": [-2, 1, 2, -1], "lrank": 2, "rrank": 2, "conj": 4,
         "dprm": [1, 2], "lprm": [1, 2], "rprm": [1, 2], "ncd": 1, "nlu": 1, "nru": 1,
         "note": "conjugated right operand switches R to the transposed layout (:5701-5709)"},
    ],
    "contractions": [
        {"name": "test_talsh_c", "cite": "TALSH/test.cpp:38-147", "dtype": "R8",
         "pattern": "D(a,b,i,j)+=L(c,b,d,a)*R(j,d,i,c)",
         "ddims": [40, 40, 20, 20], "ldims": [40, 40, 40, 40], "rdims": [20, 40, 20, 40],
         "dinit": 0.0, "linit": 0.001, "rinit": 0.01, "alpha": 2.0, "accumulative": True,
         "element": 0.032, "norm1": 20480.0},
        {"name": "test_talsh_cxx_first", "cite": "TALSH/test.cpp:190-206", "dtype": "R8",
         "pattern": "D(a,b,c,d)+=L(d,i,c,j)*R(j,b,i,a)",
         "ddims": [40, 40, 20, 20], "ldims": [20, 40, 20, 40], "rdims": [40, 40, 40, 40],
         "dinit": 1.0, "linit": 0.01, "rinit": 0.001, "alpha": 0.5, "accumulative": False,
         "element": 0.008},
        {"name": "test_talsh_cxx_second", "cite": "TALSH/test.cpp:207-216", "dtype": "R8",
         "pattern": "D(a,b,c,d)+=L(d,i,c,j)*R(j,b,i,a)",
         "ddims": [40, 40, 20, 20], "ldims": [20, 40, 20, 40], "rdims": [40, 40, 40, 40],
         "dinit": 0.008, "linit": 0.01, "rinit": 0.001, "alpha": 0.5, "accumulative": True,
         "element": 0.016},
        {"name": "test_talsh_xl_c4", "cite": "TALSH/test.cpp:310-345 (ODIM=8, VDIM=16 here)",
         "dtype": "C4", "pattern": "D(i,a,j,b)+=L(j,a,k,c)*R(k,b,i,c)",
         "ddims": [8, 16, 8, 16], "ldims": [8, 16, 8, 16], "rdims": [8, 16, 8, 16],
         "dinit": 1e-4, "linit": 0.01, "rinit": 0.001, "alpha": 0.5, "accumulative": True,
         "element": 128 * 1e-3 * 1e-2 * 0.5 + 1e-4},
        {"name": "test_talsh_xl_scalar", "cite": "TALSH/test.cpp:353-359 (ODIM=8, VDIM=16 here)",
         "dtype": "C4", "pattern": "D()+=L(i,a,j,b)*R(j,b,i,a)",
         "ddims": [], "ldims": [8, 16, 8, 16], "rdims": [8, 16, 8, 16],
         "dinit": 0.0, "linit": 0.01, "rinit": 0.001, "alpha": 1.0, "accumulative": True,
         "element": 128.0 * 128.0 * 1e-3 * 1e-2},
        {"name": "test_talsh_xlf", "cite": "TALSH/main.F90:350-412", "dtype": "R8",
         "pattern": "D(a,b,c,d)+=L(p,c,a)*R(p,b,d)",
         "ddims": [33, 33, 33, 33], "ldims": [420, 33, 33], "rdims": [420, 33, 33],
         "dinit": 1e-4, "linit": 1e-3, "rinit": 1e-2, "alpha": 0.5, "accumulative": True,
         "element": 420 * 1e-3 * 1e-2 * 0.5 + 1e-4},
        {"name": "test_nvtal_c", "cite": "TALSH/test.cpp:1016-1110", "dtype": "R8",
         "pattern": "D(a,b,c,d)+=L(d,c,k,l)*R(b,a,k,l)",
         "ddims": [40, 40, 40, 40], "ldims": [40, 40, 40, 40], "rdims": [40, 40, 40, 40],
         "dinit": 0.0, "linit": 0.01, "rinit": 0.001, "alpha": 1.0, "accumulative": True,
         "element": 1600 * 1e-5, "norm2sq": (40 ** 4) * (1600 * 1e-5) ** 2},
    ],
    "explicit_loop": {
        "cite": "TALSH/test.cpp:895-1000",
        "pattern": "D(a,b)+=L(c,d)*R(d,a,b,c)", "ddims": [2, 5], "ldims": [5, 2], "rdims": [2, 2, 5, 5],
        "alphas": [-2.0, 1.0],
        "note": "after the two contractions D = -L*R; adding L*R by explicit loops returns ~0",
    },
}


def parse_ctm(path):
    lines = [ln.strip() for ln in open(path) if ln.strip()]
    out = []
    for i in range(0, len(lines) - 1, 2):
        pat = lines[i]
        nums = [int(x) for x in lines[i + 1].split()]
        shapes, p = [], 0
        for _ in range(3):
            r = nums[p]; shapes.append(nums[p + 1:p + 1 + r]); p += 1 + r
        out.append({"pattern": pat, "ddims": shapes[0], "ldims": shapes[1], "rdims": shapes[2]})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default=os.environ.get("TALSH_REFERENCE_ROOT"),
                    help="root of the ExaTENSOR source tree (or set TALSH_REFERENCE_ROOT); "
                         "without it only kats.json is written")
    args = ap.parse_args()
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(KATS, f, indent=1)
    ctm = os.path.join(args.reference_root, "TALSH", "tensor_contractions.txt") if args.reference_root else None
    if ctm and os.path.exists(ctm):
        with open(os.path.join(HERE, "ctm_patterns.json"), "w") as f:
            json.dump({"source": "TALSH/tensor_contractions.txt", "entries": parse_ctm(ctm)}, f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
