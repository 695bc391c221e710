"""Time the reference's own CPU path (FL/legacy/FL_correction_core.py, numpy /
numba) on a bounded sample of the 128^3 x 3-element x 120-angle corrected
MLEM, and scale it to the whole job.  A recipe that reads the reference
checkout (oracle.build_ref.ref_root); it runs where that checkout is, not on
the GPU machines, and prints one JSON object.

The legacy package imports with the same stub modules as
tests/golden/make_golden.py (xraylib, skimage, ... are absent; none of them
is reached by the functions timed).  Timed, per stage of the job:

  rotation    rot3D (FL/image_util.py:165-203), scipy order 1, the 4 channels
              at one angle
  incident    cal_incident_x_ray_atten (:2010-2062) at one angle
  cone        atten_2D_slice_all_elem (:1498-1518), the per-slice body that
              cal_xrf_atten (:2065-2117) maps over a Pool of round(0.8*cores)
              workers: one slice, all 3 elements, one angle
  mlem        generate_H_jit (:2204-2279, numba prange) + mlem_matrix
              (:99-119) for one slice: the body of absorption_correction
              (:2456-2477) without its file reads, with 5 iterations (the
              k iterations between rebuilds)

usage: python oracle/time_legacy.py [N] [angles]
"""
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "tests", "golden"))


def main():
    N = int(sys.argv[1]) if len(sys.argv) > 1 else 128
    A = int(sys.argv[2]) if len(sys.argv) > 2 else 120
    L, k_iter, n_iter = 3, 5, 50
    n_rec = math.ceil(n_iter / k_iter)
    import types
    import make_golden as mg
    mg.import_reference()
    lg = types.ModuleType("FL.legacy")
    lg.__path__ = [os.path.join(mg.REF, "FL", "legacy")]
    sys.modules["FL.legacy"] = lg
    import FL.legacy.FL_correction_core as core
    import FL.image_util as iu
    from fl_correction_b200 import phantoms
    from fl_correction_b200.detector_mask import generate_detector_mask
    wl = phantoms.make_workload(1)
    frac = wl.frac()[:, :N, :N, :N].astype(np.float64)
    p = phantoms.xrf_params(wl.elements, A, 14.0, 1e-4)
    p_a = {"cs": {k: (np.asarray(v).reshape(-1)[0] if k.endswith("-x") else v)
                  for k, v in p["cs"].items()}, "rho": p["rho"], "pix": p["pix"]}
    # the legacy cone reads mask3D[str(max(n_row - i, 7))] for every row i
    ang = phantoms.cone_mask_angle(7.0, 30.0)
    core.load_global_mask({str(n): generate_detector_mask(ang, ang, n) for n in range(7, N + 1)})
    cores = os.cpu_count() or 1
    pool = max(1, round(cores * 0.8))
    out = {"job": "%d^3, %d elements, %d angles, %d MLEM iterations, rebuilt every %d"
                  % (N, L, A, n_iter, k_iter), "cores": cores, "pool_workers": pool}
    t0 = time.perf_counter()
    iu.rot3D(frac, 37.0)
    out["rotation_s_per_angle"] = time.perf_counter() - t0
    # the legacy incident term pairs compound j with element j (:2046-2048):
    # the element compounds only
    p_x = {"cs": dict(p_a["cs"], elem_compound=p["elem_compound"][:L]), "rho": p["rho"],
           "pix": p["pix"]}
    t0 = time.perf_counter()
    core.cal_incident_x_ray_atten(frac[:L], p_x)
    out["incident_s_per_angle"] = time.perf_counter() - t0
    mu = np.stack([sum(frac[j] * p["cs"][f"{c}-{e}"] * p["rho"][c]
                       for j, c in enumerate(p["elem_compound"])) for e in wl.elements])
    core.mu_all_elem = mu
    sli = N // 2
    t0 = time.perf_counter()
    core.atten_2D_slice_all_elem(sli)
    out["cone_s_per_slice_angle"] = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    atten3D = rng.uniform(0.5, 1.0, (A, N, N))
    theta = np.linspace(0, np.pi, A, endpoint=False)
    H_tot = np.zeros((A * N, N * N))
    H_zero = np.zeros((N, N * N))
    core.generate_H_jit((1, N, N), theta[:2], atten3D[:2], H_tot[:2 * N], H_zero)   # numba JIT
    t0 = time.perf_counter()
    H = core.generate_H_jit((1, N, N), theta, atten3D, H_tot, H_zero)
    out["H_s_per_slice"] = time.perf_counter() - t0
    y = H @ rng.uniform(0.0, 1.0, N * N) * 1.05
    t0 = time.perf_counter()
    core.mlem_matrix(np.ones((N, N)), H, y.copy(), k_iter)
    out["mlem_s_per_slice_block"] = time.perf_counter() - t0
    # the job: per rebuild, rotation + incident per angle and the cone per
    # slice-angle (Pool of `pool` workers); per rebuild and element, H and k
    # MLEM iterations per slice
    job = n_rec * (A * (out["rotation_s_per_angle"] + out["incident_s_per_angle"])
                   + A * N * out["cone_s_per_slice_angle"] / pool
                   + L * N * (out["H_s_per_slice"] + out["mlem_s_per_slice_block"]))
    out["job_s"] = job
    out["mlem_iters_per_s"] = n_iter / job
    print(json.dumps(out))


if __name__ == "__main__":
    main()
