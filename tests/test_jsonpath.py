"""JSONPath compiler: the reference's golden bytecode and unsupported set
(jsonpath/JSONPathParserTest.java:33-60), and agreement of the native
compiler with the oracle's restatement on a random corpus."""

from __future__ import annotations

import random

import pytest

import gpjson_b200 as gj
from oracle import jsonpath_oracle as J


def B():
    return J.ir_builder()


# JSONPathParserTest.simpleProvider (:33-44): (path, IRBuilder calls, maxDepth)
GOLDEN = [
    ("$.user.lang", B().property("user").down().property("lang").down().storeResult().end(), 2),
    ("$['user'][\"lang\"]", B().property("user").down().property("lang").down().storeResult().end(), 2),
    (
        "$.user.lang[?(@ == 'nl')]",
        B().property("user").down().property("lang").down().expressionStringEquals("nl").storeResult().end(),
        2,
    ),
    ("$[1]", B().index(1).down().storeResult().end(), 1),
    ("$['us\\'er'][\"lang\"]", B().property("us\\'er").down().property("lang").down().storeResult().end(), 2),
    (
        "$.categoryPath[1:3]",
        B().property("categoryPath").down().index(1).down().storeResult().up().index(2).down().storeResult().end(),
        2,
    ),
    (
        "$.categoryPath[1:3].id",
        B()
        .property("categoryPath").down().index(1).down().property("id").down().storeResult().up().up()
        .index(2).down().property("id").down().storeResult().end(),
        3,
    ),
    (
        "$.categoryPath[1:4].id",
        B()
        .property("categoryPath").down().index(1).down().property("id").down().storeResult().up().up()
        .index(2).down().property("id").down().storeResult().up().up()
        .index(3).down().property("id").down().storeResult().end(),
        3,
    ),
]

# JSONPathParserTest.unsupportedProvider (:54-60)
UNSUPPORTED = [
    "$.routes[*].legs[*].steps[*].distance.text",
    "$.meta.view.columns[*].name",
    "$.claims.P150[*].mainsnak.property",
]


@pytest.mark.parametrize("path,builder,depth", GOLDEN, ids=[g[0] for g in GOLDEN])
def test_golden_bytecode_oracle(path, builder, depth):
    ir, max_depth, _ = J.compile_path(path)
    assert ir == builder.toByteArray()
    assert max_depth == depth


@pytest.mark.parametrize("path,builder,depth", GOLDEN, ids=[g[0] for g in GOLDEN])
def test_golden_bytecode_native(path, builder, depth):
    c = gj.compile_path(path)
    assert c.bytecode == builder.toByteArray()
    assert c.max_depth == depth


@pytest.mark.parametrize("path", UNSUPPORTED)
def test_unsupported(path):
    with pytest.raises(J.UnsupportedJSONPathError):
        J.compile_path(path)
    with pytest.raises(gj.UnsupportedJSONPathException):
        gj.compile_path(path)


def test_num_results_counts_stores():
    assert gj.compile_path("$.a[0:3]").num_results == 3
    assert gj.compile_path("$.a").num_results == 1
    assert gj.compile_path("$[3:3]").num_results == 1  # empty range: only the final store


@pytest.mark.parametrize(
    "path,kind",
    [
        ("$", "parse"),
        ("", "parse"),
        ("x.a", "parse"),
        ("$.", "parse"),
        ("$.a b", "parse"),
        ("$.[", "parse"),
        ("$['']", "parse"),
        ("$[1:]", "parse"),
        ("$[99999999999]", "parse"),
        ("$['a'", "parse"),
        ("$[x]", "parse"),
        ("$x", "unsupported"),
        ("$..a", "unsupported"),
        ("$[1,2]", "unsupported"),
        ("$[*]", "unsupported"),
        ("$[?(@.a)]", "unsupported"),
    ],
)
def test_errors_match_oracle(path, kind):
    exc = J.UnsupportedJSONPathError if kind == "unsupported" else J.JSONPathError
    with pytest.raises(exc):
        J.compile_path(path)
    nexc = gj.UnsupportedJSONPathException if kind == "unsupported" else gj.JSONPathException
    with pytest.raises(nexc):
        gj.compile_path(path)
    if kind == "parse":  # a parse error is not reported as unsupported
        with pytest.raises(gj.JSONPathException) as ei:
            gj.compile_path(path)
        assert not isinstance(ei.value, gj.UnsupportedJSONPathException)


def _random_path(rng: random.Random) -> str:
    atoms = [
        lambda: "." + rng.choice(["a", "b", "user", "lang", "x_1", "é", "k" * rng.randint(1, 140)]),
        lambda: "['" + rng.choice(["a", "b c", "q\\'x", "ü"]) + "']",
        lambda: '["' + rng.choice(["a", 'x\\"y', "[.]"]) + '"]',
        lambda: f"[{rng.randint(0, 300)}]",
        lambda: f"[{rng.randint(0, 4)}:{rng.randint(0, 5)}]",
        lambda: "[?(@ == '" + rng.choice(["nl", "x y", ""]) + "')]",
        lambda: rng.choice(["[*]", "..a", "[1,2]", ".", "[", "]", " ", "[?(@ > 1)]", "$", "[1:", "['x"]),
    ]
    n = rng.randint(0, 6)
    return "$" + "".join(rng.choice(atoms)() for _ in range(n))


def test_native_matches_oracle_random():
    rng = random.Random(1234)
    for _ in range(3000):
        path = _random_path(rng)
        try:
            want = J.compile_path(path)
            werr = None
        except J.UnsupportedJSONPathError:
            want, werr = None, "unsupported"
        except J.JSONPathError:
            want, werr = None, "parse"
        try:
            c = gj.compile_path(path)
            got, gerr = (c.bytecode, c.max_depth, c.num_results), None
        except gj.UnsupportedJSONPathException:
            got, gerr = None, "unsupported"
        except gj.JSONPathException:
            got, gerr = None, "parse"
        assert (got, gerr) == (want, werr), path


def test_index_unions_are_an_opt_in_extension():
    """`[i,j,...]` (strictly ascending) compiles only with PATH_INDEX_UNIONS,
    to the same branches as the reference's ranges: a union of consecutive
    indices is byte-identical to the range over them."""
    with pytest.raises(gj.UnsupportedJSONPathException):
        gj.compile_path("$.a[1,2].b")
    ext = gj.PATH_INDEX_UNIONS
    for union, rng in (("$.a[1,2].b", "$.a[1:3].b"), ("$[0,1,2]", "$[0:3]"), ("$.x[4, 5].y[0,1]", "$.x[4:6].y[0:2]")):
        u, r = gj.compile_path(union, ext), gj.compile_path(rng)
        assert (u.bytecode, u.max_depth, u.num_results) == (r.bytecode, r.max_depth, r.num_results), union
    c = gj.compile_path("$.a[1,3,7].b", ext)
    assert c.num_results == 3 and c.max_depth == gj.compile_path("$.a[1:2].b").max_depth
    for bad in ("$[3,1]", "$[1,1]", "$[0,2,2]"):
        with pytest.raises(gj.UnsupportedJSONPathException):
            gj.compile_path(bad, ext)
    for bad in ("$[1,]", "$[1,x]", "$[1,2"):
        with pytest.raises(gj.JSONPathException) as ei:
            gj.compile_path(bad, ext)
        assert not isinstance(ei.value, gj.UnsupportedJSONPathException)
    # without the flag, errors and bytecode stay the reference's
    assert gj.compile_path("$.a[1:3].b", ext).bytecode == gj.compile_path("$.a[1:3].b").bytecode
