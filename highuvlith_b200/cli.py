"""Command line for the imaging configurations ``highuvlith_b200.config``
reads (the reference CLI, crates/highuvlith-cli/src/commands/):

    python -m highuvlith_b200.cli simulate --config X.toml [--image img.npy]
    python -m highuvlith_b200.cli sweep --config X.toml --focus-range -200,200,21 [--dose-range 26,34,5]
    python -m highuvlith_b200.cli optimize --config X.toml [--output mask.npy]

Each prints a JSON summary (simulate.rs, sweep.rs, optimize.rs with
method = "ilt")."""
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
    w = sub.add_parser("sweep", help="dose x focus grid of printed CD and contrast (commands/sweep.rs)")
    w.add_argument("--config", required=True)
    w.add_argument("--focus-range", required=True, help="start,stop,steps in nm")
    w.add_argument("--dose-range", default=None, help="start,stop,steps in mJ/cm^2 (default: the nominal dose)")
    w.add_argument("--kernel-build", default="host", choices=["host", "device", "device_reference_rule"])
    o = sub.add_parser("optimize", help="[optimize] method = 'ilt' on the device (commands/optimize.rs)")
    o.add_argument("--config", required=True)
    o.add_argument("--output", default=None, help="write the optimized transmission (.npy)")
    o.add_argument("--kernel-build", default="host", choices=["host", "device", "device_reference_rule"])
    a = ap.parse_args(argv)
    try:
        if a.cmd == "optimize":
            res = cfgmod.optimize_ilt(a.config, kernel_build=a.kernel_build)
            if a.output:
                np.save(a.output, res["mask_transmittance"])
            out = {k: v for k, v in res.items() if k != "mask_transmittance"}
        else:
            scene = cfgmod.load(a.config)
            for n in scene.notes:
                print(f"note: {n}", file=sys.stderr)
            if a.cmd == "sweep":
                doses = cfgmod.parse_range(a.dose_range) if a.dose_range else None
                out = cfgmod.sweep(scene, cfgmod.parse_range(a.focus_range), doses, kernel_build=a.kernel_build)
            else:
                res = cfgmod.simulate(scene, a.focus, a.dose, kernel_build=a.kernel_build)
                if a.image:
                    np.save(a.image, res["image"])
                out = {k: v for k, v in res.items() if k != "image"}
    except cfgmod.ConfigError as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
