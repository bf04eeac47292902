"""Generates the golden vectors in this directory from the reference itself.

Runs Astaroth's own host model (src/utils/modelsolver.cc, memory.cc,
modelreduce.cc, compiled unchanged by oracle/Makefile into
oracle/_ref/libastaroth_ref.so) on seeded inputs made by the product's
generator, and stores:

* ``golden.json`` -- sha256 of each input mesh, sha256 of the reference's
  periodic halo fill of it (bit-exact target), and every valid reduction of
  the integrated meshes;
* ``golden_<case>.npz`` -- the reference's interiors after 1 and 10 RK3
  steps (dt = 1e-3).

Needs the reference sources (run here, not on the GPU box):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from astaroth_b200 import CONFIG_PARAMS, info_to_dict, make_info, seeded_mesh  # noqa: E402
from oracle import oracle  # noqa: E402

CASES = {
    "n8": dict(n=8, seed=1),
    "n10x8x6": dict(n=(10, 8, 6), seed=7),
    "n12": dict(n=12, seed=2),
}
DT = 1e-3


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def valid_reductions():
    out = []
    for r in oracle.RTYPE_NAMES[:5]:
        out.append((r, [0]))
        out.append((r, [1, 2, 3]))
    for r in oracle.RTYPE_NAMES[5:]:
        out.append((r, [1, 2, 3, 0]))
    return out


def main() -> None:
    oracle.build()
    if not oracle.available("reference"):
        raise SystemExit("oracle/_ref/libastaroth_ref.so is missing: the reference sources "
                         "are needed to regenerate the golden vectors")
    meta = {"dt": DT, "params": CONFIG_PARAMS, "cases": {}}
    for name, c in CASES.items():
        info = make_info(c["n"], **CONFIG_PARAMS)
        p = info_to_dict(info)
        f0 = seeded_mesh(info, c["seed"])
        bc = f0.copy()
        oracle.periodic_bounds(bc, "reference")
        one = f0.copy()
        oracle.integrate(one, p, DT, 1, "reference")
        ten = f0.copy()
        oracle.integrate(ten, p, DT, 10, "reference")
        red = {}
        for r, h in valid_reductions():
            red[f"{r}:{','.join(map(str, h))}"] = oracle.reduce(one, r, h, "reference")
        meta["cases"][name] = {
            "n": c["n"], "seed": c["seed"], "input_sha256": sha(f0),
            "periodic_sha256": sha(bc), "reductions_after_1_step": red,
        }
        np.savez_compressed(HERE / f"golden_{name}.npz", step1=oracle.interior(one),
                            step10=oracle.interior(ten))
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    print("wrote", HERE)


if __name__ == "__main__":
    main()
