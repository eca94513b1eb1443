"""Prints the measured tensor-pipe rates of the current GPU (lt_measure_peak) as one JSON line:
FP64 mma.sync and the INT8 tcgen05 shapes (M128 N128, M128 N256, CTA pair M256 N128), each as the
best of `--repeat` single launches (burst) and after 0.5 s at the power limit (sustained), with the
SM clock read before and after.

    python -m libthom_b200.peak [--repeat 3]
"""
from __future__ import annotations

import argparse
import json
import subprocess

import libthom_b200 as lt

KINDS = {
    "fp64_mma_tflops": lt.LT_PEAK_FP64_MMA,
    "int8_m128n128_tops": lt.LT_PEAK_INT8_MMA_N128,
    "int8_m128n256_tops": lt.LT_PEAK_INT8_MMA_N256,
    "int8_pair_m256n128_tops": lt.LT_PEAK_INT8_MMA_PAIR,
}


def sm_clock_mhz():
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.sm", "--format=csv,noheader,nounits", "-i", "0"],
                             capture_output=True, text=True, timeout=10).stdout.strip()
        return float(out.splitlines()[0])
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    res = {"sm_mhz_before": sm_clock_mhz()}
    for name, kind in KINDS.items():
        vals = [lt.measure_peak(kind) / 1e12 for _ in range(args.repeat)]
        res[name] = max(vals)
        res[name + "_all"] = vals
        res[name + "_sustained"] = lt.measure_peak(kind | lt.LT_PEAK_SUSTAINED) / 1e12
    res["sm_mhz_after"] = sm_clock_mhz()
    print(json.dumps(res))


if __name__ == "__main__":
    main()
