"""Regenerates this folder's autotuner table on the GPU it runs on.

    python zig-algebra_b200/tune/make_table.py [--out PATH] [--lo 10] [--hi 24]

Times every pass shape and stage count (zntt_autotune) for both fields and
every log n in [lo, hi], and writes the table (JSON lines keyed by GPU name)
to PATH, by default b200.json beside this script.  Run it again whenever the
pass kernels change: plans and batches read the table, and a stale one picks
shapes by the old kernels' timings.
"""
from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)


def _load():
    """Imports the package from its folder (its name is not an identifier)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("zig_algebra_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["zig_algebra_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "b200.json"))
    ap.add_argument("--lo", type=int, default=10)
    ap.add_argument("--hi", type=int, default=24)
    args = ap.parse_args()
    z = _load()
    z.init(0)
    z.tune_clear()
    for F in z.FIELDS:
        z.autotune(F, args.lo, args.hi)
    z.tune_save(args.out)
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
