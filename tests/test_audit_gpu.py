"""The rational ray auditor on GPU extractions (scripts/audit_gpu.py's use):
both peelers on resolved fixtures and a generated scene, and the CLI."""

import json

import pytest
import parity

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


@pytest.mark.parametrize("method", ["events", "peel"])
@pytest.mark.parametrize("name", ["holes", "partial", "stacked", "components", "perspective_torus"])
def test_fixture_audit(name, method):
    from peel_b200 import DevicePeeler, EventPeeler
    from peel_b200.audit import audit
    from peel_b200.io import load_scene

    arrays, labels, data = load_scene(parity.fixture(name))
    p = (EventPeeler if method == "events" else DevicePeeler)(*arrays)
    p.run()
    report = audit(p, labels, data)
    assert report["rank_mismatches"] == 0, report["examples"][:3]
    assert report["checked_rays"] > 0


def test_generated_scene_audit():
    from peel_b200 import EventPeeler, scenes
    from peel_b200.audit import audit
    from peel_b200.io import scene_data

    host = scenes.nested_icospheres()
    arrays = scenes.to_device(host)
    p = EventPeeler(*arrays)
    p.run()
    report = audit(p, list(range(arrays[1].shape[0])), scene_data(*host), samples=256)
    assert report["rank_mismatches"] == 0, report["examples"][:3]
    assert report["checked_rays"] > 500


def test_cli(tmp_path, capsys):
    from peel_b200.audit import main

    path = tmp_path / "holes.json"
    path.write_text(json.dumps(parity.fixture("holes")))
    assert main([str(path), "--samples", "64"]) == 0
    report = json.loads(capsys.readouterr().out)
    assert report["rank_mismatches"] == 0 and report["checked_rays"] > 0
