"""Generate the golden fixtures used by the parity tests.

Run once in a container where the reference checkout is mounted:

    python tests/golden/make_golden.py REFERENCE_CHECKOUT

It copies two kinds of data (no code) out of the reference:

* the CC0 scene fixtures ``tests/fixtures/*.json`` and their manifest
  (``tests/fixtures/manifest.json``), the inputs the reference's own tests use
  (``tests/gpu/test_peeler.py:86-100``);
* the exact outputs the reference's CGAL solvers wrote for nine of those
  scenes (``results/examples/<name>/arrangement/exact.json``), reduced to what
  the parity tests compare: per source the exact projected polygon and affine
  depth plane (``src/camera.cpp:66-154``), and per (layer, source) the exact
  doubled region area and region rings (``src/arrangement_oracle.cpp:4-91``).

All numbers stay exact rational strings "n/d".  The output is small (a few
hundred KB) and is committed; the GPU box never reads the reference.
"""

import json
import shutil
import sys
from fractions import Fraction
from pathlib import Path

HERE = Path(__file__).resolve().parent


def area2(ring):
    """Twice the signed area of a ring of exact points (shoelace)."""
    total = Fraction(0)
    for i in range(len(ring)):
        x0, y0 = ring[i]
        x1, y1 = ring[(i + 1) % len(ring)]
        total += x0 * y1 - x1 * y0
    return total


def ring_of(raw):
    return [(Fraction(x), Fraction(y)) for x, y in raw]


def domain_area2(domain):
    total = Fraction(0)
    for piece in domain:
        total += abs(area2(ring_of(piece["outer"])))
        for hole in piece["holes"]:
            total -= abs(area2(ring_of(hole)))
    return total


def main(reference):
    reference = Path(reference)
    fixtures = HERE / "fixtures"
    fixtures.mkdir(exist_ok=True)
    manifest = json.loads((reference / "tests/fixtures/manifest.json").read_text())
    shutil.copyfile(reference / "tests/fixtures/manifest.json", fixtures / "manifest.json")
    for entry in manifest["fixtures"]:
        name = entry["name"]
        shutil.copyfile(reference / f"tests/fixtures/{name}.json", fixtures / f"{name}.json")
    expected = {}
    for path in sorted((reference / "results/examples").glob("*/arrangement/exact.json")):
        name = path.parent.parent.name
        data = json.loads(path.read_text())
        sources = [
            {
                "id": s["source_id"],
                "score": s["score"],
                "polygon": s["initial_domain"][0]["outer"] if s["initial_domain"] else [],
            }
            for s in data["sources"]
        ]
        regions = []
        for layer in data["layers"]:
            for r in layer["regions"]:
                regions.append(
                    {
                        "layer": layer["layer_index"] - 1,
                        "source": r["source_id"],
                        "area2": str(domain_area2(r["domain"])),
                        "domain": r["domain"],
                    }
                )
        expected[name] = {
            "window": data["window"],
            "camera": {k: data["camera"][k] for k in ("type", "near", "world_to_camera")},
            "sources": sources,
            "regions": regions,
            "layers": len(data["layers"]),
        }
    (HERE / "exact_regions.json").write_text(json.dumps(expected, indent=1) + "\n")
    print(f"{len(manifest['fixtures'])} fixtures, {len(expected)} exact region sets")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_CHECKOUT")
    main(sys.argv[1])
