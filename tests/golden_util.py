"""Load the golden fixtures written by tests/golden/make_golden.py."""

import functools
import json
import pathlib

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@functools.lru_cache(maxsize=None)
def load(name):
    return json.loads((GOLDEN / f"{name}.json").read_text())


def ints(xs):
    return [int(x) for x in xs]


def xor_all(xs):
    r = 0
    for x in xs:
        r ^= int(x)
    return r
