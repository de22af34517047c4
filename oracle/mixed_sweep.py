"""TEST INFRASTRUCTURE ONLY — the per-lane mixed-precision experiment on the CPU.

    python -m oracle.mixed_sweep [--devices 64] [--np 400]

The drawn J-V curves' devices (seed 20261203, half frozen after a 1.0 V pre-bias, half with free
ions) through `solve_batch` with the block sweep in FP64 and, per lane, in FP32 while the lane's
last Newton step exceeds a threshold theta (oracle/dd_cpu.cpp `ddc_solve_batch_mixed`): for each
theta the share of steps whose sweep is FP32, the steps against FP64's, the converged flags that
differ, the largest |dJ| / J scale where both converged, and the contraction of the step size
after an FP32 step (geometric mean per device; its median and largest over the devices). A
table in Markdown on stdout.
"""

from __future__ import annotations

import argparse

import numpy as np

from jaxdd_b200.workloads import V_SCAN, drawn_devices
from oracle import cpu, dd

THETAS = (1e-1, 3e-2, 1e-2, 1e-3, 1e-4, 1e-6)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--devices", type=int, default=64)
    ap.add_argument("--np", type=int, default=400)
    args = ap.parse_args()
    tree = dd.prepare(drawn_devices(args.devices, NP=args.np))
    V = np.ascontiguousarray(V_SCAN)
    J0, ok0, _, s0 = cpu.solve_batch_mixed(tree, V, -1.0)
    steps0 = s0[:, 1].sum()
    print(f"{args.devices} drawn devices, NP {args.np}, {V.size} voltages; FP64 sweep: "
          f"{int(steps0)} Newton steps, converged {ok0.mean():.4f}\n")
    print("| theta | FP32-sweep steps | steps / FP64's | flags differing | max abs(dJ)/J_scale "
          "| contraction after an FP32 step (median, largest) |")
    print("|---|---|---|---|---|---|")
    for theta in THETAS:
        J, ok, _, st = cpu.solve_batch_mixed(tree, V, theta)
        both = ok & ok0
        err = np.max(np.where(both, np.abs(J - J0), 0.0), axis=1) / tree["J_scale"]
        share = st[:, 0].sum() / st[:, :2].sum()
        contr = st[:, 2][np.isfinite(st[:, 2])]
        print(f"| {theta:g} | {share:.3f} | {st[:, :2].sum() / steps0:.3f} | "
              f"{int(np.sum(ok != ok0))} of {ok.size} | {np.max(err):.2e} | "
              f"{np.median(contr):.2e}, {np.max(contr):.2e} |")


if __name__ == "__main__":
    main()
