"""Regenerates the committed fixtures under tests/golden/.

1. graph_convert/: the reference's own graph-convert test inputs and expected
   outputs (tools/graph-convert/test-inputs/, registered by
   tools/graph-convert/CMakeLists.txt:29-31 as edgelist2gr/csv2gr followed by
   gr2edgelist and a byte comparison).  They are copied verbatim so the .gr
   conversion tests run where the reference tree is absent.
2. generators.json: digests of the seeded generators' CSR arrays at small
   sizes, so that a change to the generators (which would silently change every
   benchmark input) fails a test.

Run from the repository root:
    python tests/golden/make_golden.py [--reference PATH_TO_GALOIS_TREE]
(or set GALOIS_REFERENCE).  Without a reference tree the graph_convert/
fixtures already committed are kept and only generators.json is rewritten.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        if a is not None:
            h.update(a.tobytes())
    return h.hexdigest()[:32]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GALOIS_REFERENCE"),
                    help="root of a Galois source tree (its tools/graph-convert/test-inputs are copied)")
    args = ap.parse_args()
    out = HERE / "graph_convert"
    out.mkdir(exist_ok=True)
    REF = Path(args.reference) / "tools" / "graph-convert" / "test-inputs" if args.reference else None
    if REF is not None and REF.exists():
        for f in sorted(REF.iterdir()):
            shutil.copyfile(f, out / f.name)
    sys.path.insert(0, str(ROOT))
    from galois_b200 import assign_weights_f32, assign_weights_u32, erdos_renyi, grid2d, rmat

    gens = {}
    g, perm = rmat(12, 16, seed=20, symmetrize=True)
    gens["rmat12_sym_seed20"] = {"n": g.n, "m": g.m, "digest": digest(g.end_offs, g.col, perm)}
    g, perm = rmat(11, 16, seed=22, symmetrize=False)
    assign_weights_u32(g, 1, 255, seed=22)
    gens["rmat11_dir_seed22_w"] = {"n": g.n, "m": g.m, "digest": digest(g.end_offs, g.col, g.w_u32, perm)}
    g = grid2d(33, 47)
    gens["grid33x47"] = {"n": g.n, "m": g.m, "digest": digest(g.end_offs, g.col)}
    g = erdos_renyi(5000, 8.0, seed=3)
    assign_weights_f32(g, seed=3)
    gens["er5000_seed3_wf"] = {"n": g.n, "m": g.m, "digest": digest(g.end_offs, g.col, g.w_f32)}
    (HERE / "generators.json").write_text(json.dumps(gens, indent=1, sort_keys=True) + "\n")
    print("wrote", out, HERE / "generators.json")


if __name__ == "__main__":
    main()
