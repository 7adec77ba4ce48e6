"""Calibrates the image-parity thresholds: the oracle against itself, on the CPU.

    python tests/calibrate_parity.py [case ...] [--pairs 3]

For every case of tests/parity_cases.py the oracle renders the scene twice with independent seeds,
once at the case's GPU sample count and once at its oracle sample count, and the statistics of
tests/parity_stats.py are taken between the two, exactly as the GPU test takes them between the
GPU and the oracle. Repeated for several seed pairs; the worst value of each statistic is written
to tests/golden/parity_calibration.json, from which the GPU test sets its bars. Unbiased
estimators of the same image give these values by chance alone.
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))

import oracle  # noqa: E402
from parity_cases import BY_NAME, CASES  # noqa: E402
from parity_stats import compare, sample_variance  # noqa: E402
from toaster_b200.scene import Scene  # noqa: E402

OUT = HERE / "golden" / "parity_calibration.json"


def render(o: oracle.Oracle, spp: int, seed: int):
    mean, sq, _ = o.render(seed=seed, moments=True)
    return mean, sample_variance(mean, sq, spp)


def calibrate(case, pairs: int) -> dict:
    scene = case.make()
    g_oracle = oracle.Oracle(Scene(**{**scene.__dict__, "samples": case.gpu_spp}))
    o_oracle = oracle.Oracle(Scene(**{**scene.__dict__, "samples": case.cpu_spp}))
    worst = {}
    runs = []
    for k in range(pairs):
        t0 = time.perf_counter()
        gm, gv = render(g_oracle, case.gpu_spp, seed=1000 + 2 * k)
        om, ov = render(o_oracle, case.cpu_spp, seed=1001 + 2 * k)
        st = compare(gm, gv, case.gpu_spp, om, ov, case.cpu_spp)
        st["seconds"] = time.perf_counter() - t0
        runs.append(st)
        for key in ("outside_pixel", "outside_block", "median_z", "global_dz", "rel_mean"):
            worst[key] = max(worst.get(key, 0.0), abs(st[key]))
        print(case.name, k, json.dumps(st), flush=True)
    return {"gpu_spp": case.gpu_spp, "cpu_spp": case.cpu_spp, "pairs": pairs, "worst": worst, "runs": runs}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*")
    ap.add_argument("--pairs", type=int, default=3)
    args = ap.parse_args()
    OUT.parent.mkdir(parents=True, exist_ok=True)
    for case in [BY_NAME[n] for n in args.cases] if args.cases else CASES:
        result = calibrate(case, args.pairs)
        data = json.loads(OUT.read_text()) if OUT.exists() else {}
        data[case.name] = result
        OUT.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
