"""Time the reference's own CUDA implementation on this GPU (measurement of the
reference, not part of the product).

Runs forward::a2_fp_per_angle and backward::a2_bp_per_angle of the reference
(CT_Recon/hf_siddon_class.hpp:195-225, 313-347), built for sm_100a into
oracle/_ref/libref_gpu.so, for a few views of the 256^3 / 360-view / 512^2
workload and extrapolates to one MLEM iteration (all views).  Each call goes
through the reference's classes as its MLEM loop does per view: set-up with its
blocking step-count read-back (a_calc_initial_limits), the step-synchronous
kernels, and the copy of one view in and one result out.  The elementwise ratio
and update kernels are not included (they are a small part).

    python oracle/time_ref_gpu.py [--views 2]

prints one JSON line.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# import oracle/ as the package beside recon_b200, not its oracle.py as a module
sys.path = [os.path.dirname(_HERE)] + [p for p in sys.path if os.path.abspath(p or ".") != _HERE]

from oracle import oracle as O  # noqa: E402
from recon_b200.configs import PLAIN_GPU, geom_dict  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--views", type=int, default=2)
    a = ap.parse_args()
    R = O.ref_gpu()
    if R is None:
        print(json.dumps({"unavailable": "oracle/_ref/libref_gpu.so is not built"}))
        return
    cfg = dict(PLAIN_GPU)
    g = O.Geom.from_dict(geom_dict(cfg))
    n = int(cfg["NumProj"])
    dang = np.float32(cfg["DeltaAng"])
    rng = np.random.default_rng(0)
    vol = rng.random(g.nvox).astype(np.float32)
    img = np.zeros(g.npix, np.float32)
    bp = np.zeros(g.nvox, np.float32)
    R.ref_gpu_fp_view(g, 0.0, vol, img)  # warm-up (context, module load)
    views = [int(k * n / a.views) + n // (2 * a.views) for k in range(a.views)]
    t_fp = t_bp = 0.0
    steps = []
    for v in views:
        ang = float(np.float32(v) * dang)
        t0 = time.perf_counter()
        loopn = R.ref_gpu_fp_view(g, ang, vol, img)
        t1 = time.perf_counter()
        R.ref_gpu_bp_view(g, ang, img, bp)
        t2 = time.perf_counter()
        t_fp += t1 - t0
        t_bp += t2 - t1
        steps.append(int(loopn))
    per_view = (t_fp + t_bp) / len(views)
    print(json.dumps({"workload": "plain_gpu_256cube_360x512x512", "views_timed": views, "loopN": steps,
                      "fp_s_per_view": t_fp / len(views), "bp_s_per_view": t_bp / len(views),
                      "s_per_iteration": per_view * n, "iter_per_s": 1.0 / (per_view * n)}))


if __name__ == "__main__":
    main()
