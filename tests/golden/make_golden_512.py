"""Golden statistics of one FP64 RK3 step at 512^3, the benchmark's size,
from the reference itself: Astaroth's host model (src/utils/modelsolver.cc,
compiled unchanged into oracle/_ref/libastaroth_ref.so), run on the seeded
benchmark mesh with the benchmark physics and dt = 1e-3.

The 512^3 state (8.9 GB) is too large to commit, so this stores:

* the sha256 of the input mesh (the product's acHostMeshRandomizeSeeded and
  the oracle's generator give the same bytes);
* per field, over the interior after the step: the sum, the sum of absolute
  values, the sum of squares, the minimum and the maximum;
* the values of 1024 interior cells at seeded positions.

tests/test_gpu_fullsize.py::test_512_one_step_vs_reference_golden checks the
device's step against them.  Needs the reference sources and a few minutes of
the host model's OpenMP threads (run here, not on the GPU box):
    python tests/golden/make_golden_512.py
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402

N = 512
SEED = 2
DT = 1e-3
SAMPLES = 1024
SAMPLE_SEED = 512


def sample_positions(n: int = N):
    """(k, j, i) interior indices (0-based, without the halo) of the sampled cells."""
    rng = np.random.default_rng(SAMPLE_SEED)
    return rng.integers(0, n, size=(SAMPLES, 3))


def stats(fields: np.ndarray, n: int = N) -> dict:
    """Per-field statistics of the interior and the sampled values."""
    h = 3
    pos = sample_positions(n)
    out = {"sum": [], "sum_abs": [], "sum_sq": [], "min": [], "max": [], "samples": []}
    for q in range(8):
        a = fields[q, h:h + n, h:h + n, h:h + n]
        out["sum"].append(float(np.sum(a)))
        out["sum_abs"].append(float(np.sum(np.abs(a))))
        out["sum_sq"].append(float(np.sum(a * a)))
        out["min"].append(float(a.min()))
        out["max"].append(float(a.max()))
        out["samples"].append([float(a[k, j, i]) for k, j, i in pos])
    return out


def main() -> None:
    oracle.build()
    if not oracle.available("reference"):
        raise SystemExit("oracle/_ref/libastaroth_ref.so is missing: the reference sources "
                         "are needed to regenerate this file")
    f = oracle.seeded_mesh(N, SEED)
    meta = {"n": N, "seed": SEED, "dt": DT, "steps": 1, "params": oracle.box_params(N),
            "input_sha256": hashlib.sha256(np.ascontiguousarray(f).tobytes()).hexdigest()}
    t0 = time.time()
    oracle.integrate(f, oracle.box_params(N), DT, 1, "reference")
    meta["reference_seconds"] = round(time.time() - t0, 1)
    meta.update(stats(f))
    (HERE / "golden_512.json").write_text(json.dumps(meta) + "\n")
    print("wrote golden_512.json in", meta["reference_seconds"], "s")


if __name__ == "__main__":
    main()
