"""CPU checks of the native library: it loads, exports every declared entry
point, and its own pattern parser agrees with the oracle's restatement of
get_contr_pattern_dig on the golden fixtures, the ctm corpus and random
patterns.  No kernel runs here (there is no GPU)."""
import json
import os
import random
import re

import pytest

import exatensor_b200 as X
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def declared_functions():
    names = set()
    for h in ("talsh_b200.h", "talsh.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name.startswith(("tb_", "talsh")) and not name.endswith("_t"):
                names.add(name)
    return sorted(names)


def test_library_builds_and_loads():
    from exatensor_b200 import build
    build.build()
    assert os.path.exists(X.LIB_PATH)
    X.lib()


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    assert hasattr(X.lib(), name), name


def test_no_gpu_is_reported_not_hidden():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(X.TBError):
        X.device_init(0)


KATS = json.load(open(os.path.join(GOLD, "kats.json")))
CTM = json.load(open(os.path.join(GOLD, "ctm_patterns.json")))["entries"]


@pytest.mark.parametrize("case", KATS["patterns"], ids=lambda c: c["pattern"])
def test_product_parser_kats(case):
    cptrn, d, l, r, cj = X.parse_pattern(case["pattern"])
    assert cptrn == case["cptrn"] and [d, l, r] == case["ranks"] and cj == case["conj"]


@pytest.mark.parametrize("case", KATS["pattern_errors"], ids=lambda c: c["pattern"] or "empty")
def test_product_parser_rejects(case):
    with pytest.raises(X.TBError):
        X.parse_pattern(case["pattern"])


def test_product_parser_ctm_corpus():
    for e in CTM:
        assert X.parse_pattern(e["pattern"]) == tuple(O.parse_pattern(e["pattern"]))


def _random_pattern(rng):
    labels = [chr(ord("a") + i) for i in range(16)]
    rng.shuffle(labels)
    nc, nl, nr = rng.randint(0, 3), rng.randint(0, 3), rng.randint(0, 3)
    c, lu, ru = labels[:nc], labels[nc:nc + nl], labels[nc + nl:nc + nl + nr]
    L = c + lu; R = c + ru; D = lu + ru
    rng.shuffle(L); rng.shuffle(R); rng.shuffle(D)
    conj = rng.random() < 0.3
    return "D(%s)+=L%s(%s)*R(%s)" % (",".join(D), "+" if conj else "", ",".join(L), ",".join(R))


def test_product_parser_random_agrees_with_oracle():
    rng = random.Random(42)
    for _ in range(500):
        p = _random_pattern(rng)
        try:
            ref = O.parse_pattern(p)
        except O.PatternError:
            with pytest.raises(X.TBError):
                X.parse_pattern(p)
            continue
        assert X.parse_pattern(p) == tuple(ref), p


def test_product_parser_random_corruptions_agree_on_acceptance():
    rng = random.Random(7)
    for _ in range(500):
        p = list(_random_pattern(rng))
        for _ in range(rng.randint(1, 2)):
            i = rng.randrange(len(p))
            p[i] = rng.choice("abcz,|()+_ 9")
        p = "".join(p)
        try:
            ref = O.parse_pattern(p)
            ok = True
        except O.PatternError:
            ok = False
        if ok:
            assert X.parse_pattern(p) == tuple(ref), p
        else:
            with pytest.raises(X.TBError):
                X.parse_pattern(p)
