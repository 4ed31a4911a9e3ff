"""Extract rwig's known-answer vectors into tests/golden/tinytest_golden.json.

The reference's own tests (inst/tinytest/test_sinkhorn.R,
inst/tinytest/test_barycenter.R) hold inputs and expected outputs computed by
independent Julia/ForwardDiff restatements.  This script reads those two R files
as text (it executes nothing) and writes their numbers as JSON, so the parity
tests need no access to the reference tree at run time.

Usage:  python tests/golden/make_golden.py [path/to/rwig]
"""
from __future__ import annotations

import json
import os
import re
import sys


def _tokens(src: str):
    return re.findall(r"[A-Za-z_][A-Za-z_0-9.]*|-?\d+\.?\d*(?:[eE][-+]?\d+)?|-?\.\d+(?:[eE][-+]?\d+)?|[(),=]", src)


class _Parser:
    """Parses the R subset used by the fixtures: numbers, c(...), rbind(...), list(...)."""

    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else None

    def take(self, want=None):
        tok = self.t[self.i]
        if want is not None and tok != want:
            raise ValueError(f"expected {want!r}, got {tok!r}")
        self.i += 1
        return tok

    def value(self):
        tok = self.take()
        if tok in ("c", "rbind", "list"):
            self.take("(")
            items, names = [], []
            while self.peek() != ")":
                name = None
                if self.i + 1 < len(self.t) and self.t[self.i + 1] == "=" and re.match(r"[A-Za-z_]", self.peek()):
                    name = self.take()
                    self.take("=")
                items.append(self.value())
                names.append(name)
                if self.peek() == ",":
                    self.take(",")
            self.take(")")
            if tok == "list":
                return {n: v for n, v in zip(names, items)}
            if tok == "rbind":
                return [list(r) for r in items]  # list of rows
            return [float(x) for x in items]
        return float(tok)


def _assign(src: str, name: str):
    m = re.search(rf"^{re.escape(name)}\s*<-\s*", src, re.M)
    if not m:
        raise KeyError(name)
    p = _Parser(_tokens(src[m.end():]))
    return p.value()


def extract(ref_root: str) -> dict:
    sk = open(os.path.join(ref_root, "inst/tinytest/test_sinkhorn.R")).read()
    bc = open(os.path.join(ref_root, "inst/tinytest/test_barycenter.R")).read()
    out = {
        "source": "rwig inst/tinytest/test_sinkhorn.R, inst/tinytest/test_barycenter.R",
        "tolerance": "10*sqrt(.Machine$double.eps) (test_sinkhorn.R:4), mean relative difference",
        "sinkhorn": {
            "inputs": {"a": _assign(sk, "a"), "b": _assign(sk, "b"), "C": _assign(sk, "C"),
                       "reg": _assign(sk, "reg")},
            "vanilla": _assign(sk, "sol_jl_vanilla"),
            "log": _assign(sk, "sol_jl_log"),
        },
        "barycenter": {
            "inputs": {"A": _assign(bc, "A"), "C": _assign(bc, "C"), "w": _assign(bc, "w"),
                       "b": _assign(bc, "b"), "reg": _assign(bc, "reg")},
            "parallel": _assign(bc, "sol_jl_parallel"),
            "log": _assign(bc, "sol_jl_log"),
        },
    }
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RWIG_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_golden.py <rwig source tree>  (or set RWIG_REFERENCE_DIR)")
    data = extract(ref)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tinytest_golden.json")
    with open(dst, "w") as fh:
        json.dump(data, fh, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main()
