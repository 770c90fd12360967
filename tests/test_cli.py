"""The command line (warp_peel/__main__.py:13-77): argument errors on the CPU,
reported before any device work with argparse's exit code 2, and the written
layers.npz and sidecar on a GPU, against the exact oracle."""

import subprocess
import sys

import pytest
from conftest import ROOT

FIXTURE = ROOT / "tests/golden/fixtures/single.json"


def run(*args):
    return subprocess.run([sys.executable, "-m", "peel_b200", *map(str, args)],
                          capture_output=True, text=True, timeout=300,
                          cwd=ROOT / "exact-depth-peeling_b200")


@pytest.mark.parametrize("args,message", [
    ((FIXTURE,), "--out"),
    ((FIXTURE, "--out", "x.npz", "--method", "clip"), "invalid choice"),
    ((FIXTURE, "--out", "x.npz", "--method", "events", "--pieces", "4", "--device", "cpu"),
     "--pieces applies only to --method peel"),
])
def test_argument_errors(args, message):
    done = run(*args)
    assert done.returncode == 2
    assert message in done.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["events", "peel"])
@pytest.mark.parametrize("name", ["holes", "perspective_torus"])
def test_layers_npz_against_the_oracle(tmp_path, name, method):
    """The command line end to end on a GPU: layers.npz holds uv, world,
    external source ids and zero-based layers whose per (layer, source) areas
    are the exact oracle's, and the sidecar records the format, the method,
    the scene and the status (warp_peel/__main__.py:55-73)."""
    import json
    from collections import defaultdict

    import numpy as np
    import parity
    import torch

    from oracle import exact as ex

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    scene_path = ROOT / f"tests/golden/fixtures/{name}.json"
    out = tmp_path / "out" / "layers.npz"
    done = run(scene_path, "--out", out, "--method", method)
    assert done.returncode == 0, done.stderr
    status = json.loads(done.stdout)
    mesh = np.load(out)
    assert sorted(mesh.files) == ["layers", "sources", "uv", "world"]
    t = status["triangles"]
    assert mesh["uv"].shape == (t, 3, 2) and mesh["world"].shape == (t, 3, 3)
    assert mesh["sources"].dtype == np.int64 and mesh["layers"].dtype == np.int32
    data = parity.fixture(name)
    scene = ex.read_scene(data, resolved_mesh=True)
    layers, _ = ex.extract(scene)
    assert mesh["layers"].min() == 0 and mesh["layers"].max() == len(layers) - 1
    ids = {tri.get("id", i) for i, tri in enumerate(data["triangles"])}
    assert set(mesh["sources"].tolist()) <= ids
    area = defaultdict(float)
    for tri, source, layer in zip(mesh["uv"], mesh["sources"], mesh["layers"]):
        a, b = tri[1] - tri[0], tri[2] - tri[0]
        area[(int(layer), int(source))] += 0.5 * (a[0] * b[1] - a[1] * b[0])
    parity.assert_areas(dict(area), parity.oracle_areas(scene, layers))
    sidecar = json.loads(out.with_suffix(".json").read_text())
    assert sidecar == {"format": "warp-peel-approximate-v1", "zero_based_layers": True,
                       "exact_geometry": False, "method": method, "scene": str(scene_path),
                       "output": status}
