"""bench.py's host-side bookkeeping on CPU (no GPU, no extraction).

* every configuration the bench times has a workload description;
* the CPU legs time the overlapping 720K scene on its first layers only and
  say so in their sample text, and every other scene in full;
* the algorithmic byte count follows the stated formula (inputs plus 128 B per
  output triangle).
"""

import sys

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_timed_configurations_are_described():
    for name in ("knot-65536", bench.SECOND_CONFIG, "primitives-720k", "batched-128",
                 "icospheres-2560", "stack-65536"):
        assert name in bench.DESCRIPTIONS, name
    assert bench.SECOND_CONFIG == "overlap-720k"
    config = bench.workload_config(bench.SECOND_CONFIG, range(3), range(5))
    assert config["workload"].startswith("overlap-720k: ")
    assert (config["faces"], config["vertices"]) == (5, 3)


def test_cpu_sample_text_names_the_layer_cap():
    info = {"layers": 70, "triangles": 123}
    capped = bench.cpu_sample_text("overlap-720k", info)
    assert "first 4 layers only" in capped and "lower bound" in capped
    full = bench.cpu_sample_text("knot-65536", info)
    assert full.startswith("full extraction") and "70 layers" in full
    assert set(bench.CPU_LAYER_SAMPLE) == {"overlap-720k"}


def test_algorithmic_bytes():
    assert bench.algorithmic_bytes(10, 20, 30) == 24 * 10 + 12 * 20 + 128 + 48 + 128 * 30
