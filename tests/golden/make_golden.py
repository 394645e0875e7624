"""Generate tests/golden/templates.json from the reference's own tables.

Reads src/math/aslTemplates.cxx of the ASL sources (the velocity sets with
their laplacian and gradient coefficients; LBGK weights are LC/6 plus 1 for
the rest vector, aslTemplates.cxx:55-68) and
test/testMath/testReductionFunction.cc (the reduction known answers), and
writes them as JSON so that the CPU tests can pin the oracle and the
library's tables against the reference without the reference present.

    python tests/golden/make_golden.py /path/to/ASL
"""
import json
import re
import sys
from fractions import Fraction
from pathlib import Path


def number(tok: str) -> float:
    tok = tok.strip()
    if not re.fullmatch(r"[-+0-9./\s]+", tok):
        raise ValueError(tok)
    neg = tok.startswith("-")
    tok = tok.lstrip("+-")
    if "/" in tok:
        a, b = tok.split("/")
        v = Fraction(a.rstrip(".") or "0") / Fraction(b.rstrip(".") or "1")
    else:
        v = Fraction(tok.rstrip(".") or "0")
    return float(-v if neg else v)


def templates(src: str) -> dict:
    out = {}
    for name in ("d3q7", "d3q15", "d3q19", "d3q27"):
        mv = re.search(r"AVec<int>\s+%sDataV?\[(\d+)\]\s*=\s*\{(.*?)\};" % name, src, re.S)
        vecs = [[int(v) for v in t.split(",")] for t in re.findall(r"makeAVec\(([-\d,\s]+)\)", mv.group(2))]
        entry = {"vectors": vecs}
        for kind in ("LC", "GC"):
            mc = re.search(r"double\s+%sData%s\[\d+\]\s*=\s*\{(.*?)\};" % (name, kind), src, re.S)
            if mc:
                entry[kind.lower()] = [number(t) for t in mc.group(1).split(",")]
        out[name] = entry
    return out


def reductions(src: str) -> list:
    """The sums the reference's reduction tests check: in testSum / testSum1,
    `unsigned int n(N)` elements and `approxEqual(..., F.f*n)`."""
    out = []
    for body in re.findall(r"bool testSum\w*\(\)\s*\{(.*?)\n\}", src, re.S):
        n = re.search(r"unsigned int n\((\d+)\)", body)
        f = re.search(r"approxEqual\(summator->res\.v\(\)\[0\],\s*([\d.]+)f?\*n\)", body)
        if n and f:
            out.append({"n": int(n.group(1)), "sum": float(f.group(1).rstrip(".")) * int(n.group(1))})
    return out


def main(root: str):
    root = Path(root)
    tpl = templates((root / "src/math/aslTemplates.cxx").read_text())
    red = reductions((root / "test/testMath/testReductionFunction.cc").read_text())
    doc = {"source": "ASL src/math/aslTemplates.cxx, test/testMath/testReductionFunction.cc",
           "templates": tpl, "reduction_known_answers": red}
    out = Path(__file__).with_name("templates.json")
    out.write_text(json.dumps(doc, indent=1) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the ASL source tree>")
    main(sys.argv[1])
