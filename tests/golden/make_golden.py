"""Generates tests/golden/harmonics.json from the reference's mpmath fixtures, and
tests/golden/helmholtz_fmm3d.json from its FMM3D Helmholtz fixture (see helmholtz()).

The reference ships 40-digit mpmath values of the real solid harmonics and their
gradients (fmm-math/fixtures/harmonics_{A,B,C}.json, generator
tools/fixtures/gen_harmonics.py, seeds 20260929 / 20261001).  This script keeps a
small subset (degree-truncated, a few points per set) so the committed fixture stays
small; it is run once, in a container where the reference is mounted:

    python tests/golden/make_golden.py /path/to/reference

The degree truncation is exact: values of degree n do not depend on p
(fmm-math/src/harmonics.rs:97-98), so the leading (p+1)^2 entries of a record are the
harmonics at the smaller p.
"""
import json
import os
import sys


def truncate(rec, p, grads):
    n = (p + 1) ** 2
    out = {"x": rec["x"], "value": rec["value"][:n]}
    if grads and "grad" in rec:
        out["grad"] = [g[:n] for g in rec["grad"]]
    return out


def main(ref):
    fx = os.path.join(ref, "fmm-math", "fixtures")
    sets = []
    plan = [("A", 12, 4, True), ("B", 8, 8, True), ("C", 16, 4, False)]
    for name, p, count, grads in plan:
        with open(os.path.join(fx, f"harmonics_{name}.json")) as f:
            d = json.load(f)
        entry = {"set": name, "p": p, "seed": d["header"]["seed"], "regular": [], "irregular": []}
        for fam in ("regular", "irregular"):
            for rec in d.get(fam, [])[:count]:
                entry[fam].append(truncate(rec, p, grads))
        sets.append(entry)
    out = {
        "source": "fmm-math/fixtures/harmonics_{A,B,C}.json of tbetcke/fmm (mpmath, 40 digits, "
        "17 significant digits of the nearest double)",
        "sets": sets,
    }
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "harmonics.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


def helmholtz(ref):
    """tests/golden/helmholtz_fmm3d.json: FMM3D v2.1.0's Helmholtz direct sum (h3ddirectcg,
    with 1/(4 pi)) from fmm-ref/fixtures/helmholtz_fmm3d.json (generator
    tools/fixtures/gen_helmholtz_fmm3d.py, seed 20261028): every source, target and charge,
    and for seven of the twelve cases the values at the 40 targets and the first 40
    sources (the fixture's points are the sources, then the targets)."""
    with open(os.path.join(ref, "fmm-ref", "fixtures", "helmholtz_fmm3d.json")) as f:
        d = json.load(f)
    ns = len(d["sources"])
    keep = list(range(40)) + list(range(ns, ns + len(d["targets"])))
    cases = []
    for i in (0, 1, 3, 5, 7, 9, 11):
        c = d["cases"][i]
        cases.append({"label": c["label"], "k": c["k"], "charges": c["charges"], "points": keep,
                      "potential": [c["potential"][j] for j in keep],
                      "gradient": [c["gradient"][j] for j in keep]})
    out = {
        "source": "fmm-ref/fixtures/helmholtz_fmm3d.json of tbetcke/fmm (FMM3D v2.1.0 h3ddirectcg, "
        "17 significant digits; e^{ikr}/(4 pi r); gradient [re x, im x, re y, im y, re z, im z])",
        "sources": d["sources"], "targets": d["targets"], "charges": d["charges"], "cases": cases,
    }
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "helmholtz_fmm3d.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    reference = sys.argv[1]
    main(reference)
    helmholtz(reference)
