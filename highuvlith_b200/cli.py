"""Command line: ``python -m highuvlith_b200.cli simulate --config X.toml``
(the reference CLI's simulate command, crates/highuvlith-cli/src/commands/
simulate.rs, for the imaging configurations ``highuvlith_b200.config``
reads).  Prints a JSON summary; ``--image`` saves the aerial image (.npy)."""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from . import config as cfgmod


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="highuvlith_b200.cli")
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("simulate", help="aerial image, contrast, printed CD and NILS at one dose/focus")
    s.add_argument("--config", required=True)
    s.add_argument("--focus", type=float, default=None, help="focus override (nm)")
    s.add_argument("--dose", type=float, default=None, help="dose override (mJ/cm^2)")
    s.add_argument("--image", default=None, help="write the aerial image as .npy")
    s.add_argument("--kernel-build", default="host", choices=["host", "device", "device_reference_rule"])
    a = ap.parse_args(argv)
    try:
        scene = cfgmod.load(a.config)
    except cfgmod.ConfigError as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
    for n in scene.notes:
        print(f"note: {n}", file=sys.stderr)
    res = cfgmod.simulate(scene, a.focus, a.dose, kernel_build=a.kernel_build)
    if a.image:
        np.save(a.image, res["image"])
    out = {k: v for k, v in res.items() if k != "image"}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
