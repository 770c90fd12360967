"""Learned pool sizing for the EventPeeler.

The reference sizes every pool at worst case from the face count
(warp_peel/events.py:19-33, ``EventCapacities.for_mesh``: 4N frontier, 8N
regions, 32N hits, vertices and triangles).  Here a 16 -> 64 -> 64 -> 3
perceptron predicts, for each of the 16 x 16 screen tiles, the extraction's
output fragments, triangles and depth layers from sixteen cheap projection
features (``edp_tile_features``), and the sums size the pools:

* regions = frontier = m_F * sum(F)
* triangles = m_T * sum(T), boundary vertices = triangles + 2 * regions
  (a polygon of n vertices gives n fan triangles, a triangle gives one)
* hits = m_H * sum(F * L)  (a ray group holds at most one hit per layer)
* layers = m_L * max(L)

with margins m fixed from the training set, and none above the worst-case
sizing.  Fragment and triangle counts are learned per 4,096 faces, with the
count features scaled alike, so the network trained on 4K-64K-face meshes
sizes finer meshes of the same kind.  An extraction that overflows a
learned pool reruns with ``EventCapacities.for_mesh`` (``peel``), so the
outputs never depend on the prediction; only the memory does.

Every network operation runs in this library's own CUDA kernels:
``edp_mlp_infer`` (tensor cores, BF16 weights, FP32 accumulation),
``edp_mlp_grad`` (forward and backward) and ``edp_adam_step``.

    python -m peel_b200.learned train --meshes 2000 --out pool_sizing.json

trains on the counts the peeler itself produces on seeded meshes
(``scenes.training_mesh``, seeds 1000 upward) and writes the weights,
feature normalisation and margins (the 99th percentile over the training
meshes of actual / predicted, plus 5%; the other 1% fall back).
"""

import argparse
import json
import math
import time
from dataclasses import replace
from pathlib import Path

import numpy as np

from . import _lib
from .events import EventCapacities, EventPeeler

WEIGHTS = Path(__file__).resolve().parent / "pool_sizing.json"
TILE_AXIS, INPUTS, HIDDEN, OUTPUTS, PARAMS = 16, 16, 64, 3, 5443
TILES = TILE_AXIS * TILE_AXIS
SCRATCH = TILES * 12 + 4
TARGETS = ("fragments", "triangles", "layers")
PER_FACES = 4096  # fragment and triangle counts are learned per 4,096 faces
FORMAT = "peel-b200-pool-sizing-v2"  # features and targets per PER_FACES faces


def per_faces(counts, faces, inverse=False):
    """Counts [tiles, 3] with fragments and triangles taken per PER_FACES
    faces (or back, with `inverse`); layers are left as they are."""
    out = np.array(counts, dtype=np.float64, copy=True)
    scale = PER_FACES / max(int(faces), 1)
    out[:, :2] = out[:, :2] / scale if inverse else out[:, :2] * scale
    return out
# Offsets of the parameter blocks (edp.h): W1, b1, W2, b2, W3, b3.
SLICES = {"W1": (0, (HIDDEN, INPUTS)), "b1": (1024, (HIDDEN,)), "W2": (1088, (HIDDEN, HIDDEN)),
          "b2": (5184, (HIDDEN,)), "W3": (5248, (OUTPUTS, HIDDEN)), "b3": (5440, (OUTPUTS,))}


def _stream(device):
    import torch

    return torch.cuda.current_stream(device).cuda_stream


def init_params(seed=0):
    """He-initialised parameters (float64 numpy, the layout of edp.h)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS)
    for name, (at, shape) in SLICES.items():
        if name.startswith("W"):
            fan_in = shape[1]
            p[at:at + shape[0] * shape[1]] = rng.normal(0, math.sqrt(2.0 / fan_in),
                                                        size=shape).ravel()
    return p


def unpack(p):
    """{name: array} views of a flat parameter vector."""
    return {name: np.asarray(p)[at:at + int(np.prod(shape))].reshape(shape)
            for name, (at, shape) in SLICES.items()}


def tile_features(arrays):
    """[tiles, 16] float32 device tensor of a mesh (vertices, faces, camera,
    settings device tensors)."""
    import torch

    vertices, faces, camera, settings = arrays
    device = vertices.device
    scratch = torch.empty(SCRATCH, dtype=torch.float32, device=device)
    features = torch.empty((TILES, INPUTS), dtype=torch.float32, device=device)
    with torch.cuda.device(device):
        _lib.check(_lib.load().edp_tile_features(
            vertices.data_ptr(), vertices.shape[0], faces.data_ptr(), faces.shape[0],
            camera.data_ptr(), settings.data_ptr(), scratch.data_ptr(), features.data_ptr(),
            _stream(device)), "tile features")
    return features


def infer(params, x):
    """Network outputs [rows, 3] (float32 device tensor) of feature rows x."""
    import torch

    x = x.contiguous()
    y = torch.empty((x.shape[0], OUTPUTS), dtype=torch.float32, device=x.device)
    with torch.cuda.device(x.device):
        _lib.check(_lib.load().edp_mlp_infer(params.data_ptr(), x.data_ptr(), x.shape[0],
                                             y.data_ptr(), _stream(x.device)), "mlp infer")
    return y


def gradient(params, x, target, mask, scale):
    """(gradient [PARAMS], loss) of sum(mask (y - target)^2) * scale, from the
    training kernel (float32 device tensors)."""
    import torch

    grad = torch.zeros(PARAMS, dtype=torch.float32, device=x.device)
    loss = torch.zeros(1, dtype=torch.float32, device=x.device)
    with torch.cuda.device(x.device):
        _lib.check(_lib.load().edp_mlp_grad(
            params.data_ptr(), x.contiguous().data_ptr(), target.contiguous().data_ptr(),
            mask.contiguous().data_ptr(), x.shape[0], float(scale), grad.data_ptr(),
            loss.data_ptr(), _stream(x.device)), "mlp gradient")
    return grad, loss


def tile_targets(peeler):
    """[tiles, 3] counts of a finished extraction: output fragments (by the
    polygon's vertex mean), triangles (by centroid) and layers (one more than
    the deepest polygon layer) per screen tile."""
    info = peeler.read_status()
    count = info["polygons"]
    n = peeler.output.sizes[:count].cpu().numpy()
    v = peeler.output.vertices[:count].cpu().numpy()
    layers = peeler.output_layers[:count].cpu().numpy()
    live = n >= 3
    idx = np.arange(v.shape[1])[None, :] < n[:, None]
    centre = (v * idx[:, :, None]).sum(1) / np.maximum(n, 1)[:, None]

    def tile(uv):
        c = np.clip(np.floor(uv * TILE_AXIS).astype(np.int64), 0, TILE_AXIS - 1)
        return c[:, 1] * TILE_AXIS + c[:, 0]

    out = np.zeros((TILES, OUTPUTS))
    pt = tile(centre[live])
    np.add.at(out[:, 0], pt, 1.0)
    np.maximum.at(out[:, 2], pt, layers[live] + 1.0)
    t = info["triangles"]
    tri = peeler.triangles_uv[:t].cpu().numpy()
    np.add.at(out[:, 1], tile(tri.mean(1)), 1.0)
    return out


class PoolSizer:
    """Capacities from the trained network (``WEIGHTS`` by default)."""

    def __init__(self, path=WEIGHTS, device="cuda"):
        import torch

        data = json.loads(Path(path).read_text())
        if data.get("format") != FORMAT:
            raise ValueError(f"{path}: weights in format {data.get('format')!r}, "
                             f"expected {FORMAT!r} (retrain with `python -m peel_b200.learned "
                             "train`)")
        self.meta = data
        self.params = torch.tensor(data["params"], dtype=torch.float32, device=device)
        self.mean = torch.tensor(data["feature_mean"], dtype=torch.float32, device=device)
        self.std = torch.tensor(data["feature_std"], dtype=torch.float32, device=device)
        self.margins = data["margins"]

    def predict(self, arrays):
        """[tiles, 3] predicted counts (host numpy)."""
        x = (tile_features(arrays) - self.mean) / self.std
        y = infer(self.params, x).double().cpu().numpy()
        return per_faces(np.expm1(np.clip(y, 0.0, 30.0)), arrays[1].shape[0], inverse=True)

    def capacities(self, arrays, scale=1.0):
        """EventCapacities for a mesh; `scale` multiplies the prediction (a
        test uses it to force an under-estimate)."""
        counts = self.predict(arrays) * scale
        return capacities_from_counts(counts, self.margins, arrays[1].shape[0])


def capacities_from_counts(counts, margins, faces):
    """EventCapacities from per-tile counts [tiles, 3] (fragments, triangles,
    layers) and the margins; no pool exceeds the worst-case sizing's."""
    base = EventCapacities.for_mesh(faces)
    fragments, triangles, layers = counts[:, 0], counts[:, 1], counts[:, 2]
    regions = int(margins["fragments"] * fragments.sum()) + 256
    tris = int(margins["triangles"] * triangles.sum()) + 1024
    hits = int(margins["hits"] * (fragments * np.maximum(layers, 1.0)).sum()) + 1024
    depth = int(margins["layers"] * layers.max(initial=1.0)) + 8
    return replace(base, frontier=min(base.frontier, regions), regions=min(base.regions, regions),
                   hits=min(base.hits, hits), vertices=min(base.vertices, tris + 2 * regions),
                   triangles=min(base.triangles, tris), layers=min(base.layers, depth))


OVERFLOW = 2 | 4 | 8 | 16 | 32 | 64 | 1024 | 2048  # pool-capacity bits of status[9]


def peel(arrays, sizer=None, scale=1.0, **options):
    """Extract with learned pools; on a pool overflow, extract again with the
    conservative ``EventCapacities.for_mesh`` pools, doubled where even they
    overflow (``sizing.fit_event_capacities``).  Returns (peeler, capacities,
    fell_back)."""
    from .sizing import fit_event_capacities

    sizer = sizer or PoolSizer(device=arrays[0].device)
    cap = sizer.capacities(arrays, scale)
    p = EventPeeler(*arrays, capacities=cap, **options)
    p.run()
    p.stream.synchronize()
    if int(p.status[9].item()) & OVERFLOW:
        del p
        p, cap = fit_event_capacities(arrays, EventCapacities.for_mesh(arrays[1].shape[0]),
                                      headroom=1.0, **options)
        return p, cap, True
    return p, cap, False


def workspace_bytes(peeler):
    """Device bytes a peeler's workspace holds."""
    out = np.zeros(1, dtype=np.int64)
    _lib.check(_lib.load().edp_workspace_bytes(peeler._ws.handle, out.ctypes.data),
               "workspace bytes")
    return int(out[0])


# ---------------------------------------------------------------- training

def _generate(seed):
    from . import scenes

    return scenes.training_mesh(seed)


def dataset(seeds, device="cuda", processes=None):
    """(features [M, tiles, 16], targets [M, tiles, 3]) numpy arrays of the
    meshes of `seeds`, each peeled with pools that fit it (sizing.py).  The
    meshes are generated by a pool of spawned processes."""
    import multiprocessing
    import os

    from . import scenes
    from .sizing import fit_event_capacities

    processes = processes or min(16, os.cpu_count() or 1)
    with multiprocessing.get_context("spawn").Pool(processes) as pool:
        meshes = pool.map(_generate, list(seeds), chunksize=4)
    feats, targs = [], []
    for host in meshes:
        arrays = scenes.to_device(host, device)
        p, _ = fit_event_capacities(arrays, headroom=1.0)
        info = p.read_status()  # raises on a failed extraction
        feats.append(tile_features(arrays).cpu().numpy())
        raw = tile_targets(p)
        assert raw[:, 1].sum() == info["triangles"]
        targs.append(per_faces(raw, len(host[1])))
        del p
    return np.stack(feats), np.stack(targs)


def train(features, targets, epochs=60, batch=4096, lr=3e-3, seed=0, device="cuda", log=None):
    """Adam on log(1 + count) targets with a cosine learning-rate decay;
    returns (params float32 device tensor, normalisation mean, std,
    per-epoch mean squared errors)."""
    import torch

    x = features.reshape(-1, INPUTS).astype(np.float32)
    y = np.log1p(targets.reshape(-1, OUTPUTS)).astype(np.float32)
    mean, std = x.mean(0), x.std(0) + 1e-6
    xs = torch.tensor((x - mean) / std, device=device)
    ys = torch.tensor(y, device=device)
    ms = torch.ones_like(ys)
    params = torch.tensor(init_params(seed), dtype=torch.float32, device=device)
    m1, m2 = torch.zeros_like(params), torch.zeros_like(params)
    grad = torch.zeros_like(params)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    lib = _lib.load()
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    stream = _stream(xs.device)
    step, history = 0, []
    rows = xs.shape[0]
    for epoch in range(epochs):
        order = torch.randperm(rows, device=device, generator=gen)
        loss.zero_()
        rate = lr * 0.5 * (1 + math.cos(math.pi * epoch / epochs))
        for start in range(0, rows, batch):
            idx = order[start:start + batch]
            xb, yb, mb = xs[idx].contiguous(), ys[idx].contiguous(), ms[idx].contiguous()
            _lib.check(lib.edp_mlp_grad(params.data_ptr(), xb.data_ptr(), yb.data_ptr(),
                                        mb.data_ptr(), xb.shape[0], 1.0 / (xb.shape[0] * OUTPUTS),
                                        grad.data_ptr(), loss.data_ptr(), stream), "mlp gradient")
            step += 1
            _lib.check(lib.edp_adam_step(params.data_ptr(), grad.data_ptr(), m1.data_ptr(),
                                         m2.data_ptr(), PARAMS, rate, 0.9, 0.999, 1e-8, step,
                                         stream), "adam")
        history.append(float(loss.item()) / (rows * OUTPUTS))
        if log:
            log(f"epoch {epoch}: mse {history[-1]:.5f}")
    return params, mean, std, history


def coverage_ratios(params, mean, std, features, targets, device="cuda"):
    """Per mesh, actual / predicted for each sized quantity (fragments,
    triangles, hits = sum F*L, layers = max L): {name: array}."""
    import torch

    m = torch.tensor(mean, device=device)
    s = torch.tensor(std, device=device)
    out = {"fragments": [], "triangles": [], "hits": [], "layers": []}
    for f, t in zip(features, targets):
        x = (torch.tensor(f, device=device) - m) / s
        c = np.expm1(np.clip(infer(params, x).double().cpu().numpy(), 0.0, 30.0))
        out["fragments"].append(t[:, 0].sum() / max(c[:, 0].sum(), 1.0))
        out["triangles"].append(t[:, 1].sum() / max(c[:, 1].sum(), 1.0))
        out["hits"].append((t[:, 0] * np.maximum(t[:, 2], 1)).sum()
                           / max((c[:, 0] * np.maximum(c[:, 2], 1)).sum(), 1.0))
        out["layers"].append(t[:, 2].max() / max(c[:, 2].max(), 1.0))
    return {k: np.asarray(v) for k, v in out.items()}


def margins_for(ratios, quantile=0.99, slack=1.05):
    """Margins under which the `quantile` of the training meshes' actual
    counts are covered (with `slack`); the rest fall back to the worst-case
    sizing.  Returns (margins, {name: distribution summary})."""
    margins, summary = {}, {}
    for k, r in ratios.items():
        margins[k] = float(max(1.0, np.quantile(r, quantile)) * slack)
        summary[k] = {q: float(np.quantile(r, v)) for q, v in
                      (("min", 0.0), ("median", 0.5), ("p90", 0.9), ("p99", 0.99),
                       ("max", 1.0))}
    covered = np.ones(len(next(iter(ratios.values()))), bool)
    for k, r in ratios.items():
        covered &= r <= margins[k]
    summary["covered_share"] = float(covered.mean())
    return margins, summary


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__,
                                     formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = parser.add_subparsers(dest="command", required=True)
    t = sub.add_parser("train", help="generate the training set on the GPU and train")
    t.add_argument("--meshes", type=int, default=2000)
    t.add_argument("--first-seed", type=int, default=1000)
    t.add_argument("--epochs", type=int, default=60)
    t.add_argument("--out", type=Path, default=WEIGHTS)
    args = parser.parse_args(argv)
    start = time.time()
    seeds = range(args.first_seed, args.first_seed + args.meshes)
    features, targets = dataset(seeds)
    made = time.time()
    params, mean, std, history = train(features, targets, epochs=args.epochs, log=print)
    trained = time.time()
    ratios = coverage_ratios(params, mean, std, features, targets)
    margins, distribution = margins_for(ratios)
    args.out.write_text(json.dumps({
        "format": FORMAT,
        "layout": "W1[64][16], b1[64], W2[64][64], b2[64], W3[3][64], b3[3]; weights applied "
                  "as BF16, float32 master values stored",
        "targets": ["log1p(" + name + " per tile)" for name in TARGETS],
        "tile_axis": TILE_AXIS,
        "training": {"meshes": args.meshes, "seeds": [seeds.start, seeds.stop - 1],
                     "generator": "scenes.training_mesh", "epochs": args.epochs,
                     "first_mse": history[0], "final_mse": history[-1],
                     "dataset_seconds": made - start, "training_seconds": trained - made},
        "feature_mean": [float(v) for v in mean],
        "feature_std": [float(v) for v in std],
        "margins": margins,
        "coverage": {"quantile": 0.99, "slack": 1.05, "actual_over_predicted": distribution},
        "params": [float(v) for v in params.cpu().numpy()],
    }) + "\n")
    print(json.dumps({"out": str(args.out), "final_mse": history[-1], "margins": margins,
                      "coverage": distribution, "dataset_s": made - start,
                      "train_s": trained - made}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
