"""Benchmark: self-absorption-corrected XRF MLEM on B200.

Workload (default): 128^3 volume, 3 elements (Fe, Ni, Cu), 120 angles over
0-180 deg, seeded Voronoi phantom, cone mask of a 7 mm detector at 30 mm; one
step = the full corrected reconstruction: 50 MLEM iterations with the
attenuation maps (rotation, incident scan, cone path sum) recomputed on the
device from the current estimate every 5 iterations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  `value` = MLEM iterations per second of the whole job
(all ranks), timed with CUDA events on the launching stream after W warm-up
steps; `e2e` is the same metric through the host-buffer entry point
(projections copied host->device and the result device->host inside the
timed region).  Under torchrun every rank reconstructs its own seeded volume
(replicas, weak scaling); the timing is the max over ranks.

--impl reference times the reference algorithm on the host cores through the
FP64 C restatement (oracle/), on a bounded sample of the same job that is
scaled to the full job (the sample is described in the output line).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLEM iters/s & corrected-proj GB/s (% HBM peak), batched/adjoint vs plain GPU"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 3, 4],
                   help="0/1: corrected MLEM (1 is the benchmark); 2/4: gradient "
                        "reconstruction; 3: batched uneven volumes")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-parity", action="store_true",
                   help="skip the parity leg (errors of the result against the reference's "
                        "kernels and the FP64 oracle)")
    p.add_argument("--no-ref-gpu", action="store_true",
                   help="skip timing the reference's own CUDA kernels on this GPU")
    p.add_argument("--adam-steps", type=int, default=0,
                   help="configurations 2/4: Adam steps timed (default 200 / 3)")
    p.add_argument("--case", default=None, choices=["cone", "cone_direct", "mlem", "fwd", "bwd", "stage",
                                                    "mlem_multi", "bwd_large", "grad",
                                                    "xrf_adjoint_large"],
                   help="run one kernel on a profiling-sized case instead of the benchmark")
    p.add_argument("--case-slices", type=int, default=16,
                   help="slices of 128^2 in the projector / MLEM cases (128: the benchmark's shape)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# algorithmic work counts
# ---------------------------------------------------------------------------
def sens_bytes(A, S, H, W, R=1):
    """Bytes of the sensitivity P^T 1 of one element at the reference API
    boundary: the attenuation read and the sensitivity written."""
    return 4 * (A * S * H * W + R * S * H * W)


def mlem_bytes_per_iter(A, S, H, W, R=1):
    """Bytes of one MLEM iteration of one element at the reference API
    boundary: forward (atten, C, Pf) + backward (atten, ratio, out) + the
    elementwise update (C, back, sens read; Huber neighbours; C write)."""
    fwd = 4 * (A * S * H * W + R * S * H * W + A * S * W)
    bwd = 4 * (A * S * H * W + A * S * W + R * S * H * W)
    upd = 4 * 4 * R * S * H * W
    return fwd + bwd + upd


# DRAM bytes measured by ncu: the spectral cone's five kernels move 54.3 MB
# per 128^3 volume (325.8 MB read + write for 6 volumes); an MLEM iteration
# at the benchmark's shape (120 angles x 128 slices of 128^2, one element)
# moves 1.026 GB in the lean forward and 1.023 GB in the lean backward,
# 1.018 bytes per attenuation byte.
CONE_DRAM_BYTES_PER_VOLUME = 325.8e6 / 6
MLEM_DRAM_PER_ATTEN_BYTE = (1.026144e9 + 1.023237e9) / (2 * 120 * 128 * 128 * 128 * 4)
# FP32 FMA rate measured on this pool's B200 (a chain-of-FMAs probe over
# 148 x 8 CTAs of 256 threads)
FP32_PEAK_TFLOPS = 72.5


def smooth_even(n):
    """Smallest even m >= n whose only prime factors are 2, 3 and 5 (the
    spectral cone's transform lengths)."""
    m = n + (n & 1)
    while True:
        k = m
        for r in (2, 3, 5):
            while k % r == 0:
                k //= r
        if k == 1:
            return m
        m += 2


def spectral_cone_flops(Z, X, Y, Mz, Mx, My):
    """FLOPs of the spectral cone for one volume: the depth correlation
    (8 per complex multiply-add, every frequency of every target plane and
    depth inside the volume) and the 2-D transforms (5 N log2 N per complex
    transform of length N; rows in pairs, then the half-spectrum columns),
    forward and inverse."""
    hz, hy = Mz // 2, My // 2
    Nz = smooth_even(Z + max(1, hz, Mz - 1 - hz))
    Ny = smooth_even(Y + max(hy, My - 1 - hy))
    Nyh = Ny // 2 + 1
    pairs = sum(min(Mx, X - x) for x in range(X))
    corr = 8.0 * Nz * Nyh * pairs
    plane = ((Z + 1) // 2) * 5 * Ny * np.log2(Ny) + Nyh * 5 * Nz * np.log2(Nz)
    return corr + 2 * X * plane, (Nz, Ny)


def cone_work(mask, Z, H, W):
    """(nnz-form MACs, separable MACs) of one cone volume (Z, H, W) with mask
    (Mz, Mx, My), counting only taps that land inside the volume."""
    m = np.asarray(mask, np.float64)
    Mz, Mx, My = m.shape
    hz, hy = Mz // 2, My // 2
    zc = np.array([max(0, Z - abs(dz - hz)) for dz in range(Mz)], np.float64)
    yc = np.array([max(0, H - abs(dy - hy)) for dy in range(My)], np.float64)
    nnz = 0.0
    sep = 0.0
    for dx in range(min(Mx, W)):
        xc = W - dx
        p = m[:, dx, :] != 0
        nnz += xc * float((p * zc[:, None] * yc[None, :]).sum())
        # separable: per output, taps of the y filter + taps of the z filter
        wz = int(p.any(axis=1).sum())
        wy = int(p.any(axis=0).sum())
        if wz and wy:
            sep += xc * Z * H * (wz + wy)
    return nnz, sep


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def build_problem(cfg, rank, device):
    import torch
    from fl_correction_b200 import phantoms
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.recon import CorrectedMLEM
    wl = phantoms.make_workload(cfg, seed=20240611 + 1000 * rank)
    N = wl.N
    mask = generate_detector_mask(wl.mask_angle, wl.mask_angle, N)
    solver = CorrectedMLEM(wl.param, wl.angles, mask, (N, N, N), device=device)
    truth = torch.from_numpy(wl.conc).to(device)
    solver.recompute_attenuation(truth)
    I = solver.project(truth)                       # (L, A, S, W)
    if wl.noise_max_counts:
        g = torch.Generator(device=device).manual_seed(wl.seed)
        scale = wl.noise_max_counts / float(I.max())
        I = torch.poisson(I * scale, generator=g) / scale
    torch.cuda.synchronize()
    return wl, mask, solver, I.contiguous()


def max_over_ranks(ms, world, device):
    """The maximum over ranks of a per-rank device time (every rank gets it)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def job_rate(world, iters_per_rank, ms_max):
    """Whole-job MLEM iterations per second: every rank runs its own replica of
    the workload, so the job does world x iters_per_rank in the slowest
    rank's time."""
    return world * iters_per_rank / (ms_max * 1e-3)


def run_ours(args, rank, world, device):
    import torch
    import torch.distributed as dist
    from fl_correction_b200 import _lib
    hbm, peak_kind = peaks()
    wl, mask, solver, I = build_problem(args.config, rank, device)
    N, L, A = wl.N, len(wl.elements), len(wl.angles)
    n_iter, k = wl.n_iter, wl.recompute_every

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        solver.run(I, n_iter=n_iter, recompute_every=k)
    torch.cuda.synchronize()

    # ---- timed region: K full jobs, device resident ---------------------
    cone_ev, mlem_ev = [], []
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    launches0 = _lib.query("flc_launch_count")
    with Clocks(torch.cuda.current_device()) as clk:
        start.record()
        for _ in range(args.steps):
            C = solver.run(I, n_iter=n_iter, recompute_every=k, cone_events=cone_ev,
                           mlem_events=mlem_ev)
        end.record()
        torch.cuda.synchronize()
    barrier()
    launches = _lib.query("flc_launch_count") - launches0
    ms = start.elapsed_time(end)
    t_cone = sum(a.elapsed_time(b) for a, b, _ in cone_ev)
    t_mlem = sum(a.elapsed_time(b) for a, b, _ in mlem_ev)
    ms_max = max_over_ranks(ms, world, device)

    # ---- end to end through the host-buffer entry point ----------------
    I_host = I.cpu().pin_memory()
    for _ in range(1):
        solver.run_host(I_host, n_iter=n_iter, recompute_every=k)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        out_host = solver.run_host(I_host, n_iter=n_iter, recompute_every=k)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, device)

    # ---- derived figures ----------------------------------------------
    n_cone = sum(v for _, _, v in cone_ev)
    nnz, sep = cone_work(mask.astype(np.float32), N, N, N)
    spec, nz_ny = spectral_cone_flops(N, N, N, *mask.shape)
    cone_launches = len(cone_ev)
    cone_avg_ms = t_cone / max(cone_launches, 1)
    vols_per_launch = n_cone / max(cone_launches, 1)
    fp32_peak = FP32_PEAK_TFLOPS
    mlem_iters = sum(v for _, _, v in mlem_ev)      # element-iterations timed
    bytes_it = mlem_bytes_per_iter(A, N, N, N)
    # the MLEM windows also hold the sensitivity max(P^T 1, 1e-6) that every
    # mlem call computes first (atten_cuda.cpp:283-345): one backward of
    # ratio 1 (attenuation read, sensitivity written) per element and rebuild
    n_sens = -(-n_iter // k) * L * args.steps
    bytes_sens = sens_bytes(A, N, N, N)
    mlem_bytes = bytes_it * mlem_iters + bytes_sens * n_sens
    proj_gbs = mlem_bytes / (t_mlem * 1e-3) / 1e9 if t_mlem else None
    value = job_rate(world, n_iter * args.steps, ms_max)
    e2e_value = job_rate(world, n_iter * args.steps, e2e_ms)
    cone_share = t_cone / ms if ms else 0.0
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "MLEM iters/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded phantom; no dataset ships with the reference)",
        "config": {"workload": wl.name, "volume": [N, N, N], "elements": wl.elements,
                   "angles": A, "mlem_iters": n_iter, "recompute_every": k,
                   "incident": "own-compound (FL/core.py:80-81)",
                   "mask": list(mask.shape), "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (attenuation %.1f GB per step)" % (L * A * N ** 3 * 4 / 1e9)},
        "corrected_proj_gbs": round(proj_gbs, 1) if proj_gbs else None,
        # the same metric without the amortised attenuation rebuilds: MLEM
        # iterations (all elements, their sensitivity passes included) per
        # second of rank 0's MLEM windows alone, times the replicas
        "mlem_iters_per_s_without_rebuilds": round(world * n_iter * args.steps / (t_mlem * 1e-3), 3)
                                             if t_mlem else None,
        "corrected_proj_pct_hbm": round(100 * proj_gbs / hbm, 1) if proj_gbs else None,
        "time_share": {"cone (spectral, 5 kernels per launch)": round(cone_share, 3),
                       "mlem (sensitivity + iterations)": round(t_mlem / ms, 3) if ms else None},
        # the dominant kernel: the fused MLEM iteration (with the sensitivity
        # backward of each attenuation rebuild)
        "roofline": {
            "kernel": "MLEM iteration: proj_fwd2_kernel (+ ratio) and proj_bwd2_kernel (+ update), "
                      "with the sensitivity backward of each rebuild", "bound": "hbm",
            "achieved": round(proj_gbs, 1) if proj_gbs else None, "peak": hbm, "unit": "GB/s",
            "frac": round(proj_gbs / hbm, 3) if proj_gbs else None,
            "traffic": round(MLEM_DRAM_PER_ATTEN_BYTE * 2 * A * N ** 3 * 4),
            "traffic_note": "per element-iteration: ncu dram read + write of the lean forward and backward "
                            "at this shape (the attenuation is read twice)",
            "peak_kind": peak_kind,
            "algorithmic_unit": "%.4g B per element-iteration (fwd + bwd + update at the reference API "
                                "boundary) and %.4g B per sensitivity pass (one per element and "
                                "rebuild, %d timed)" % (bytes_it, bytes_sens, n_sens),
        },
        "roofline_cone": {
            "kernel": "spectral cone (fft_filter, fft_fwd, fft_corr, fft_inv, fft_apply)",
            "bound": "fp32",
            "achieved": round(spec * vols_per_launch / (cone_avg_ms * 1e-3) / 1e12, 2),
            "peak": round(fp32_peak, 1),
            "unit": "TFLOP/s",
            "frac": round(spec * vols_per_launch / (cone_avg_ms * 1e-3) / 1e12 / fp32_peak, 3),
            "traffic": round(CONE_DRAM_BYTES_PER_VOLUME * vols_per_launch * (N / 128) ** 3),
            "traffic_note": "ncu dram read+write of the five kernels on 6 volumes of 128^3, per volume, times volumes per launch",
            "peak_kind": "measured FP32 FMA rate (chain-of-FMAs probe on this pool's B200)",
            "algorithmic_unit": "spectral FLOPs (depth correlation + 2-D FFTs, %dx%d padded planes) = %.3g per volume"
                                % (nz_ny[0], nz_ny[1], spec),
            "launches": cone_launches, "avg_ms": round(cone_avg_ms, 4),
            "separable_equivalent_tflops": round(2 * sep * vols_per_launch / (cone_avg_ms * 1e-3) / 1e12, 1),
        },
        "e2e": {"value": round(e2e_value, 3), "unit": "MLEM iters/s",
                "h2d_bytes_per_step": int(I_host.numel() * 4),
                "d2h_bytes_per_step": int(out_host.numel() * 4)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    return line


# ---------------------------------------------------------------------------
# checker legs (after the timed regions, rank 0 at N=1): the error of the
# benchmarked result, and the reference's own CUDA kernels timed beside ours
# ---------------------------------------------------------------------------
REF_SO = os.path.join(ROOT, "oracle", "_ref", "ref_atten_cuda.so")


def load_reference_extension():
    """The reference's own CUDA extension (FL/cuda_lib, built from its
    sources into oracle/_ref), or None when it was not built."""
    if not os.path.exists(REF_SO):
        return None
    from oracle.build_ref import load_built
    return load_built()


def parity_leg(wl, mask, solver, I, device):
    """Errors of this library's corrected MLEM against independent compositions
    (tests/compose.py), on inputs identical to the benchmark's:

    * first block of the benchmark (128^3, 3 elements, 120 angles; the
      attenuation built from the start value, then 5 MLEM iterations), all
      slices, against the reference's own kernels (cal_atten_cuda,
      mlem_cuda_batch) driven by the reference's torch steps, FP32 on this GPU;
    * the same block against the FP64 oracle on the centre slice (the
      oracle runs the slab of slices the cone couples to it);
    * the whole 64^3 x 60-angle workload (20 iterations, rebuilt every 5,
      Poisson noise) against the reference's kernels.
    Errors: max|a-b|/max|b| and the pointwise max |a-b|/|b| over voxels with
    |b| >= 1e-2 max|b|."""
    import torch
    from tests import compose
    from fl_correction_b200.recon import CorrectedMLEM
    from fl_correction_b200.detector_mask import generate_detector_mask
    log = lambda *a: print("[parity]", *a, file=sys.stderr, flush=True)  # noqa: E731
    out = {"bar": "1e-4 after 20 MLEM iterations, 1e-5 for maps and projections (max|a-b|/max|b|)"}
    N, L = wl.N, len(wl.elements)
    k = wl.recompute_every
    fixed = torch.ones((1, N, N, N), device=device)
    t0 = time.perf_counter()
    C1 = solver.run(I, n_iter=k, recompute_every=k)
    torch.cuda.synchronize()
    C1h = C1.cpu().numpy()
    ref = load_reference_extension()
    if ref is not None:
        Cr = compose.reference_corrected_mlem(ref, wl.param, wl.angles, mask, I, fixed, k, k)
        torch.cuda.synchronize()
        out["block1_vs_reference_kernels"] = compose.relative_errors(C1h, Cr.cpu().numpy())
        del Cr
        log("block 1 vs reference kernels", out["block1_vs_reference_kernels"],
            "%.1f s" % (time.perf_counter() - t0))
    else:
        out["block1_vs_reference_kernels"] = {"unavailable": "oracle/_ref not built"}
    # FP64 oracle on slice z of the first block: slab [z - hz, z + 1 + hz)
    t0 = time.perf_counter()
    hz = mask.shape[0] // 2
    z = N // 2
    lo, hi = max(0, z - hz), min(N, z + 1 + hz)
    Ih = I[:, :, lo:hi].cpu().numpy()
    Co = compose.oracle_corrected_mlem(wl.param, wl.angles, mask, Ih, np.ones((1, hi - lo, N, N)),
                                       k, k, z_range=(z - lo, z - lo + 1))
    out["block1_vs_fp64_oracle"] = dict(compose.relative_errors(C1h[:, z:z + 1],
                                                                Co[:, z - lo:z - lo + 1]),
                                        slices=[z, z + 1])
    log("block 1 vs oracle", out["block1_vs_fp64_oracle"], "%.1f s" % (time.perf_counter() - t0))
    del C1
    # the whole small workload against the reference's kernels
    if ref is not None:
        t0 = time.perf_counter()
        w0 = __import__("fl_correction_b200.phantoms", fromlist=["x"]).make_workload(0)
        N0 = w0.N
        m0 = generate_detector_mask(w0.mask_angle, w0.mask_angle, N0)
        s0 = CorrectedMLEM(w0.param, w0.angles, m0, (N0, N0, N0), device=device)
        truth = torch.from_numpy(w0.conc).to(device)
        s0.recompute_attenuation(truth)
        I0 = s0.project(truth)
        g = torch.Generator(device=device).manual_seed(w0.seed)
        sc = w0.noise_max_counts / float(I0.max())
        I0 = (torch.poisson(I0 * sc, generator=g) / sc).contiguous()
        C0 = s0.run(I0, n_iter=w0.n_iter, recompute_every=w0.recompute_every)
        Cr0 = compose.reference_corrected_mlem(ref, w0.param, w0.angles, m0, I0,
                                               torch.ones((1, N0, N0, N0), device=device),
                                               w0.n_iter, w0.recompute_every)
        out["cfg0_full_schedule_vs_reference_kernels"] = dict(
            compose.relative_errors(C0.cpu().numpy(), Cr0.cpu().numpy()), workload=w0.name)
        log("cfg0 vs reference kernels", out["cfg0_full_schedule_vs_reference_kernels"],
            "%.1f s" % (time.perf_counter() - t0))
    return out


def reference_gpu_leg(device, N=128, A=120, n_vol=30):
    """CUDA-event times of the reference's own kernels (FL/cuda_lib compiled
    from its sources for sm_100a) beside this library's drop-ins, through the
    same Python API, at the benchmark's shapes: the cone path sum of one
    30-volume attenuation chunk, the batched forward and backward projector
    (120 angles x 128 slices of 128^2, one reference) and 5 MLEM iterations."""
    import torch
    from fl_correction_b200.cuda_lib import atten_cuda as AC
    from fl_correction_b200.detector_mask import generate_detector_mask
    ref = load_reference_extension()
    if ref is None:
        return {"unavailable": "oracle/_ref not built"}
    g = torch.Generator(device=device).manual_seed(11)
    mask = torch.from_numpy(generate_detector_mask(13.309, 13.309, N).astype(np.float32)).to(device)
    mu = torch.rand((n_vol, N, N, N), device=device, generator=g) * 0.02
    atten = torch.rand((A, N, N, N), device=device, generator=g)
    C = torch.rand((1, N, N, N), device=device, generator=g)
    em = torch.full((A, 1), 0.02, device=device)
    th = torch.linspace(0, math.pi, A + 1, device=device)[:-1].contiguous()
    ratio = torch.rand((A, N, N), device=device, generator=g)
    I = AC.forward_emission_batch(atten, C, em, th) * 1.05

    def ev_ms(fn, reps, warm=1):
        # warm-up calls first: a GPU left idle (the host-side legs before this
        # one) runs its first kernels at low clocks
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    cases = {
        "cal_atten_cuda (%d volumes of %d^3, mask %s)" % (n_vol, N, list(mask.shape)):
            (lambda: ref.cal_atten_cuda(mu, mask), lambda: AC.cal_atten_cuda(mu, mask), 1),
        "forward_emission_batch (%d angles x %d slices of %d^2)" % (A, N, N):
            (lambda: ref.forward_emission_batch(atten, C, em, th),
             lambda: AC.forward_emission_batch(atten, C, em, th), 3),
        "backward_emission_batch (%d angles x %d slices of %d^2)" % (A, N, N):
            (lambda: ref.backward_emission_batch(atten, ratio, em, th),
             lambda: AC.backward_emission_batch(atten, ratio, em, th), 3),
        "mlem_cuda_batch (5 iterations, beta 0)":
            (lambda: ref.mlem_cuda_batch(C, atten, em, th, I, 5, 0.0, 0.01),
             lambda: AC.mlem_cuda_batch(C, atten, em, th, I, 5, 0.0, 0.01), 1),
    }
    from fl_correction_b200 import _lib
    out = {}
    for name, (fr, fo, reps) in cases.items():
        # ours first, then the reference, each warmed up and timed on its own
        # (ours: three warm-up calls and at least five timed; the reference's
        # slowest call takes about a second, so it keeps one warm-up call)
        l0 = _lib.query("flc_launch_count")
        o_reps = max(reps, 5)
        o_ms = ev_ms(fo, o_reps, warm=3)
        launches = (_lib.query("flc_launch_count") - l0) // (o_reps + 3)
        r_ms = ev_ms(fr, reps)
        out[name] = {"reference_ms": round(r_ms, 3), "ours_ms": round(o_ms, 3),
                     "speedup": round(r_ms / o_ms, 2), "ours_launches_per_call": int(launches)}
        print("[ref-gpu]", name, out[name], file=sys.stderr, flush=True)
    return out


# ---------------------------------------------------------------------------
# CPU reference (oracle port on the host cores)
# ---------------------------------------------------------------------------
def cpu_sample(cfg):
    """Time a bounded sample of the full job with the FP64 C restatement and
    scale it to the full job.  Returns (iters_per_s, description, cores)."""
    from oracle import oracle as O
    from fl_correction_b200 import phantoms
    from fl_correction_b200.core import atten_coefficients
    from fl_correction_b200.detector_mask import generate_detector_mask
    wl = phantoms.make_workload(cfg)
    N, L, A = wl.N, len(wl.elements), len(wl.angles)
    frac = wl.frac()
    n_ch = frac.shape[0]
    cx, cf = atten_coefficients(wl.param, A, n_ch)
    mask = generate_detector_mask(wl.mask_angle, wl.mask_angle, N)
    rng = np.random.default_rng(0)
    cores = O.max_threads()
    n_rec = math.ceil(wl.n_iter / wl.recompute_every)
    # (1) rotation + mu assembly + incident scan for n_st angles, all slices
    n_st = 4
    t0 = time.perf_counter()
    for a in range(n_st):
        th = wl.angles[7 + a] / 180 * math.pi
        fr = O.rotate(frac, th)
        mux = fr * cx[7 + a][:, None, None, None]
        O.incident_scan(mux[:L])
        muf = np.einsum("ij,jshw->ishw", cf[7 + a].astype(np.float64), fr)
    t_stage = (time.perf_counter() - t0) / n_st
    # (2) cone path sum for zs of N output slices of one line at one angle
    zs = max(1, N // 8)
    t0 = time.perf_counter()
    O.cone_beam_slab(muf[:1], mask, N // 2, N // 2 + zs)
    t_cone = time.perf_counter() - t0
    # (3) one MLEM iteration of one element on Bs of N slices
    Bs = max(1, N // 4)
    atten = rng.random((A, Bs, N, N))
    C = rng.random((1, Bs, N, N))
    em = np.full((A, 1), 0.02)
    thetas = (wl.angles / 180 * math.pi).astype(np.float32)
    t0 = time.perf_counter()
    Pf = O.fwd_emission(atten, C, em, thetas)
    ratio = 1.0 / np.maximum(Pf, 1e-6)
    back = O.bwd_emission(atten, ratio, em, thetas)
    O.huber_grad(C, 0.01)
    _ = C * back
    t_mlem = time.perf_counter() - t0
    job = (n_rec * (A * t_stage + L * A * (N / zs) * t_cone)
           + wl.n_iter * L * (N / Bs) * t_mlem)
    desc = ("oracle port (FP64 C, OpenMP %d threads) timed on: rotation+mu+incident scan of all "
            "%d channels (%.3f s per angle), cone path sum of %d/%d slices of 1 line at 1 angle "
            "(%.3f s), 1 MLEM iteration of 1 element on %d/%d slices (%.3f s); scaled linearly to "
            "the full job (%d recomputes x %d angles x %d lines, %d iterations x %d elements): "
            "%.1f s" % (cores, n_ch, t_stage, zs, N, t_cone, Bs, N, t_mlem, n_rec, A, L, wl.n_iter, L, job))
    return wl.n_iter / job, desc, cores, wl


def run_reference(args):
    steps = []
    desc = cores = wl = None
    for _ in range(max(1, args.steps)):
        v, desc, cores, wl = cpu_sample(args.config)
        steps.append(v)
    value = statistics.median(steps)
    return {
        "impl": "reference",
        "metric": METRIC, "value": round(value, 6), "unit": "MLEM iters/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(wl.n_iter / value * 1e3, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "volume": [wl.N] * 3, "elements": wl.elements,
                   "angles": len(wl.angles), "mlem_iters": wl.n_iter,
                   "recompute_every": wl.recompute_every},
        "cpu_baseline": {"value": round(value, 6), "unit": "MLEM iters/s", "cores": cores,
                         "kind": "port", "sample": desc},
        "e2e": {"value": round(value, 6), "unit": "MLEM iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def param_at_angles(param, n_angle, idx):
    """The parameter dict restricted to the angles idx: every per-angle array
    (length n_angle) is indexed, everything else is kept."""
    def sel(v):
        if isinstance(v, dict):
            return {k: sel(x) for k, x in v.items()}
        a = np.asarray(v) if isinstance(v, (list, np.ndarray)) else None
        if a is not None and a.dtype.kind in "fiu" and a.ndim >= 1 and a.shape[0] == n_angle:
            return a[idx]
        return v
    return sel(param)


def run_grad(args, device):
    """Configurations 2 and 4: gradient reconstruction through the attenuation.

    Reports Adam steps per second (each step: a corrected projection with the
    attenuation rebuilt per angle chunk, and its hand-written adjoint), the
    device-memory high-water mark, the gradient check, and the same step done
    the plain way: torch autograd through a torch-operator composition of the
    model (grid_sample, cumprod, conv3d, gathers) on the same GPU.  The
    gradient check compares, on a subset of the angles, the adjoint gradient
    with FP64 torch autograd and with FP64 central differences (eps = 1e-4)
    at random voxels."""
    import torch
    from fl_correction_b200 import _lib, phantoms
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.grad_recon import GradientRecon, gradient_loss
    from fl_correction_b200 import torch_composition as TM
    wl = phantoms.make_workload(args.config)
    N, L, A = wl.N, len(wl.elements), len(wl.angles)
    mask = generate_detector_mask(wl.mask_angle, wl.mask_angle, N)
    frac = wl.frac()
    torch.cuda.reset_peak_memory_stats(device)
    rec = GradientRecon(wl.param, wl.angles, mask, (N, N, N), fixed_frac=frac[L:],
                        tv_weight=1e-3, lr=1e-2, device=device)
    truth = torch.from_numpy(wl.conc).to(device)
    I = rec.proj.project(truth)
    C0 = torch.full_like(truth, 0.5)
    n_steps = args.adam_steps if args.adam_steps > 0 else (200 if args.config == 2 else 3)

    # ---- gradient check on a subset of angles ---------------------------
    sub = np.linspace(0, A - 1, 2 if N > 128 else 6).astype(int)
    chk = GradientRecon(param_at_angles(wl.param, A, sub), wl.angles[sub], mask, (N, N, N),
                        fixed_frac=frac[L:], tv_weight=1e-3, device=device)
    Ichk = I[:, sub].contiguous()
    Cc = (0.8 * truth + 0.1).contiguous()
    g32, _ = chk.gradient(Cc, Ichk)
    pr = chk.proj
    th, cx, cf, em = (pr.theta.cpu().numpy(), pr.coef_x.cpu().numpy(), pr.coef_f.cpu().numpy(),
                      pr.em.cpu().numpy())
    fixed64 = torch.from_numpy(frac[L:]).to(device, torch.float64)
    I64 = Ichk.double()

    def loss64(C):
        Pf = TM.xrf_project(torch.cat([C, fixed64]), th, cx, cf, mask, em)
        return torch.mean((Pf - I64) ** 2) / torch.mean(I64 ** 2) + 1e-3 * gradient_loss(C)

    grad_check = {"angles": int(len(sub))}
    log = lambda *a: print("[grad]", *a, file=sys.stderr, flush=True)  # noqa: E731
    log("gradient check on", len(sub), "angles")
    if N <= 128:
        # (at 256^3 the FP64 graph of even a few angles would need ~1 TB)
        C64 = Cc.double().clone().requires_grad_(True)
        loss64(C64).backward()
        grad_check["max_rel_err_vs_torch_fp64_autograd"] = float(
            (g32.double() - C64.grad).abs().max() / C64.grad.abs().max())
        del C64
    with torch.no_grad():
        Pf64 = TM.xrf_project(torch.cat([Cc.double(), fixed64]), th, cx, cf, mask, em)
        Pf32 = pr.project(Cc).double()
        grad_check["projection_max_rel_err_vs_fp64"] = float((Pf32 - Pf64).abs().max() /
                                                             Pf64.abs().max())
    del Pf64, Pf32
    # directional derivative along a random unit direction v: <g32, v> against
    # the FP64 central difference of the loss (two FP64 evaluations, so it runs
    # at every volume size)
    with torch.no_grad():
        gv = torch.Generator(device=device).manual_seed(3)
        v = torch.randn(Cc.shape, generator=gv, device=device, dtype=torch.float64)
        v /= v.norm()
        eps = 1e-3
        fd = (float(loss64(Cc.double() + eps * v)) - float(loss64(Cc.double() - eps * v))) / (2 * eps)
        ad = float((g32.double() * v).sum())
        # rel_err_over_norms: the difference against |g32| |v| (the dot product
        # sums terms of both signs, so |fd| can be far below that scale)
        grad_check["directional_fd"] = {"adjoint": ad, "fp64_central_difference": fd,
                                        "rel_err": abs(ad - fd) / abs(fd),
                                        "rel_err_over_norms": abs(ad - fd) / float(g32.double().norm())}
        del v
    log("FP64 comparison done", grad_check)
    if N <= 128:
        rng = np.random.default_rng(7)
        eps, errs = 1e-4, []
        gmax = float(g32.abs().max())
        with torch.no_grad():
            for _ in range(64):
                idx = tuple(int(rng.integers(0, n)) for n in Cc.shape)
                Cp = Cc.double().clone()
                Cm = Cp.clone()
                Cp[idx] += eps
                Cm[idx] -= eps
                fd = (float(loss64(Cp)) - float(loss64(Cm))) / (2 * eps)
                errs.append(abs(float(g32[idx]) - fd) / gmax)
        grad_check["fd_voxels"] = 64
        grad_check["max_abs_err_vs_fd_over_max_grad"] = float(max(errs))
    del chk
    torch.cuda.empty_cache()
    log("check done", grad_check)

    # ---- Adam steps ---------------------------------------------------------
    torch.cuda.reset_peak_memory_stats(device)
    rec.run(I, C0, n_steps=max(1, args.warmup))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = _lib.query("flc_launch_count")
    e0.record()
    C = rec.run(I, C0, n_steps=n_steps)
    e1.record()
    torch.cuda.synchronize()
    launches = _lib.query("flc_launch_count") - launches0
    ms = e0.elapsed_time(e1)
    misfit = float(torch.mean((rec.proj.project(C) - I) ** 2) / torch.mean(I ** 2))
    peak_gb = torch.cuda.max_memory_allocated(device) / 1e9

    log("adam: %d steps in %.1f ms" % (n_steps, ms))
    # ---- the plain way: torch autograd through the operator composition (FP32)
    plain = None
    if N <= 128:
        try:
            thf = rec.proj.theta.cpu().numpy()
            cxf, cff, emf = (rec.proj.coef_x.cpu().numpy(), rec.proj.coef_f.cpu().numpy(),
                             rec.proj.em.cpu().numpy())
            fixed32 = torch.from_numpy(frac[L:]).to(device)
            g0, _ = rec.gradient(C0, I)
            Cp = C0.clone().requires_grad_(True)
            norm = float(torch.mean(I ** 2)) * I.numel()
            n_chunk = 6                      # angles per autograd graph (memory)

            def plain_step():
                # the loss is a sum over angles: one graph per chunk of angles,
                # gradients accumulated in Cp.grad
                Cp.grad = None
                for a0 in range(0, A, n_chunk):
                    sl = slice(a0, min(A, a0 + n_chunk))
                    Pf = TM.xrf_project(torch.cat([Cp, fixed32]), thf[sl], cxf[sl], cff[sl], mask,
                                        emf[:, sl])
                    (torch.sum((Pf - I[:, sl]) ** 2) / norm).backward()
                (1e-3 * gradient_loss(Cp)).backward()

            plain_step()
            torch.cuda.synchronize()
            p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            p0.record()
            plain_step()
            p1.record()
            torch.cuda.synchronize()
            plain = {"ms_per_step": round(p0.elapsed_time(p1), 2),
                     "speedup_of_adjoint": round(p0.elapsed_time(p1) / (ms / n_steps), 2),
                     "how": "torch autograd (grid_sample, cumprod, separable conv3d, gathers) "
                            "in FP32, %d angles per graph" % n_chunk,
                     "grad_max_rel_diff_vs_adjoint": float(
                         (Cp.grad - g0).abs().max() / g0.abs().max())}
        except RuntimeError as e:   # e.g. out of memory for the stored graph
            plain = {"unavailable": str(e).splitlines()[0][:200]}
    return {
        "metric": "Adam steps/s (gradient reconstruction through the attenuation)",
        "value": round(n_steps / (ms * 1e-3), 3), "unit": "steps/s", "n_gpus": 1,
        "steps": n_steps, "warmup": args.warmup, "ms_per_step": round(ms / n_steps, 3),
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "volume": [N] * 3, "elements": wl.elements, "angles": A,
                   "loss": "mean((P(C)-I)^2)/mean(I^2) + 1e-3 TV", "optimizer": "Adam lr 1e-2"},
        "relative_misfit_after": misfit,
        "memory_high_water_gb": round(peak_gb, 2),
        "materialised_attenuation_gb": round(L * A * N ** 3 * 4 / 1e9, 1),
        "gradient_check": grad_check,
        "plain_torch_autograd": plain,
        "gpu_launches": int(launches),
    }


def run_batch(args, device):
    """Configuration 3: 16 uneven volumes (N from {64..192}, 1-3 elements,
    60-180 angles, energy and detector distance drawn per volume), the
    corrected MLEM of all of them as one CUDA graph replay with per-shape
    autotuned launch shapes, against the plain loop over volumes."""
    import torch
    from fl_correction_b200 import _lib, phantoms
    from fl_correction_b200.batch import BatchedMLEM, problems_from_workloads
    log = lambda *a: print("[batch]", *a, file=sys.stderr, flush=True)  # noqa: E731
    n_iter, k = 20, 5
    ws = phantoms.make_batch_workloads(16, n_iter=n_iter, recompute_every=k)
    log("workloads", [w.name for w in ws])
    probs = problems_from_workloads(ws, device)
    b = BatchedMLEM(probs, n_iter=n_iter, recompute_every=k, n_streams=4, autotune=True,
                    device=device)
    log("autotuned", b.knobs)
    for _ in range(max(1, args.warmup)):
        b.run_loop()
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ll0 = _lib.query("flc_launch_count")
    e[0].record()
    for _ in range(args.steps):
        loop = b.run_loop()
    e[1].record()
    loop_launches = _lib.query("flc_launch_count") - ll0
    torch.cuda.synchronize()
    loop = [c.clone() for c in loop]
    b.capture()
    for _ in range(max(1, args.warmup)):
        b.run()
    torch.cuda.synchronize()
    e[2].record()
    for _ in range(args.steps):
        out = b.run()
    e[3].record()
    torch.cuda.synchronize()
    t_loop, t_graph = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
    err = max(float((o - r).abs().max() / r.abs().max()) for o, r in zip(out, loop))
    graph_out = [c.clone() for c in out]
    # the persistent form: one launch per MLEM iteration for all 16 volumes'
    # (volume, element) problems, the schedule replayed as a CUDA graph
    b.capture_persistent()
    for _ in range(max(1, args.warmup)):
        b.run_persistent()
    torch.cuda.synchronize()
    ep = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ep[0].record()
    for _ in range(args.steps):
        pout = b.run_persistent()
    ep[1].record()
    torch.cuda.synchronize()
    t_pers = ep[0].elapsed_time(ep[1])
    err_p = max(float((o - r).abs().max() / r.abs().max()) for o, r in zip(pout, loop))
    del graph_out
    vol_iters = len(ws) * n_iter * args.steps
    return {
        "metric": "batched corrected MLEM: volume-iterations/s (16 uneven volumes)",
        "value": round(vol_iters / (t_graph * 1e-3), 3), "unit": "volume-iters/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_graph / args.steps, 2),
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "cfg3-16-uneven", "volumes": [w.name for w in ws],
                   "mlem_iters": n_iter, "recompute_every": k, "streams": len(b.groups)},
        "plain_loop": {"value": round(vol_iters / (t_loop * 1e-3), 3),
                       "ms_per_step": round(t_loop / args.steps, 2)},
        "speedup_vs_plain_loop": round(t_loop / t_graph, 3),
        "max_rel_err_vs_plain_loop": err,
        "persistent": {"value": round(vol_iters / (t_pers * 1e-3), 3),
                       "ms_per_step": round(t_pers / args.steps, 2),
                       "speedup_vs_plain_loop": round(t_loop / t_pers, 3),
                       "max_rel_err_vs_plain_loop": err_p,
                       "form": "one flc_mlem_multi_sizes call per MLEM iteration over all "
                               "(volume, element) problems (one queue launch per slice width); "
                               "attenuation rebuilt per volume; the schedule replayed as one "
                               "CUDA graph"},
        # a replay runs the kernels the eager loop launches (the graph was
        # captured from the same schedule); the host-side counter does not see
        # graph replays, so the loop's count stands for them
        "gpu_launches": int(loop_launches),
    }


def run_case(args):
    """One kernel on a profiling-sized case (for ncu): W warm-up launches, then
    one more.  cone: the fluorescence cone of one pipeline chunk at the
    benchmark size (2 angles x 3 lines of 128^3), spectral form (cone_direct:
    the direct separable kernel); mlem: one fused MLEM
    iteration (plus the sensitivity pass) at 24 angles x 16 slices of 128^2;
    fwd / bwd: the projector at 120 angles x 16 slices of 128^2; bwd_large:
    the backward at 180 angles x --case-slices slices of 256^2; grad: one
    gradient (projection + adjoint) of configuration 2; xrf_adjoint_large: the
    corrected-projection adjoint of 4 lines at 4 angles (one chunk) over
    --case-slices slices of 256^2 (the rotation adjoint in row bands)."""
    import torch
    from fl_correction_b200 import _lib
    from fl_correction_b200.cuda_lib import atten_cuda as AC
    from fl_correction_b200.detector_mask import factor_mask, generate_detector_mask
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(0)
    N = 128
    if args.case in ("cone", "cone_direct"):
        n_a, L, A = 2, 3, 120
        mask = generate_detector_mask(13.309, 13.309, N)
        u, v = (torch.from_numpy(x).to(dev) for x in factor_mask(mask))
        mu = torch.rand((n_a, L, N, N, N), device=dev, generator=g) * 0.01
        atten = torch.ones((L, A, N, N, N), device=dev)
        nb = _lib.query("flc_cone_fft_workspace_bytes", n_a * L, N, N, N, *mask.shape)
        ws = _lib.workspace(nb, dev) if args.case == "cone" else None
        def once():
            _lib.call("flc_cone_atten_apply_ws", _lib.ptr(mu), _lib.ptr(u), _lib.ptr(v),
                      _lib.ptr(atten), n_a, L, N, N, N, A, 0, *mask.shape, _lib.ptr(ws), nb,
                      _lib.stream())
    elif args.case == "mlem_multi":
        # one persistent MLEM iteration over 3 elements (the benchmark's MLEM shape
        # with --case-slices 128)
        A, B = 120, args.case_slices
        ats = [torch.rand((A, B, N, N), device=dev, generator=g) for _ in range(3)]
        em = torch.full((A, 1), 0.02, device=dev)
        th = torch.linspace(0, math.pi, A + 1, device=dev)[:-1].contiguous()
        Cs = [torch.ones((1, B, N, N), device=dev) for _ in range(3)]
        Is = [AC.forward_emission_batch(a, c * 0.7, em, th) for a, c in zip(ats, Cs)]
        box = {}
        def once():
            box["ws"] = _lib.mlem_multi(Cs, ats, [em] * 3, [th] * 3, Is, 1, 0.0, 0.01,
                                        box.get("ws"))
    elif args.case == "mlem":
        A, B = 24, 16
        atten = torch.rand((A, B, N, N), device=dev, generator=g)
        em = torch.full((A, 1), 0.02, device=dev)
        th = torch.linspace(0, math.pi, A + 1, device=dev)[:-1].contiguous()
        C0 = torch.ones((1, B, N, N), device=dev)
        I = AC.forward_emission_batch(atten, C0 * 0.7, em, th)
        def once():
            AC.mlem_cuda_batch(C0, atten, em, th, I, 1)
    elif args.case == "stage":
        # the rotation / mu / incident stage of one chunk: 10 angles x 3 lines, 4 channels, 128^3
        n_ch, L, A, n_a = 4, 3, 120, 10
        frac = torch.rand((n_ch, N, N, N), device=dev, generator=g)
        th = torch.linspace(0, math.pi, A + 1, device=dev)[:-1].contiguous()
        cx = torch.full((A, n_ch), 0.01, device=dev)
        cf = torch.full((A, L, n_ch), 0.01, device=dev)
        atten = torch.empty((L, A, N, N, N), device=dev)
        ws = torch.empty((n_a, L, N, N, N), device=dev)
        nb = _lib.query("flc_atten_stage_workspace_bytes", n_ch, N, N, N)
        ws4 = _lib.workspace(nb, dev)
        def once():
            _lib.call("flc_atten_stage_ws", _lib.ptr(frac), _lib.ptr(th), _lib.ptr(cx),
                      _lib.ptr(cf), _lib.ptr(atten), _lib.ptr(ws), n_ch, N, N, N, A, L, 0, n_a,
                      0, 1, _lib.ptr(ws4), nb, _lib.stream())
    elif args.case == "grad":
        # one gradient step of configuration 2 (96^3, 3 elements, 90 angles):
        # the corrected projection and its adjoint through mu
        from fl_correction_b200 import phantoms
        from fl_correction_b200.grad_recon import GradientRecon
        wl = phantoms.make_workload(2)
        Ng, Lg = wl.N, len(wl.elements)
        maskg = generate_detector_mask(wl.mask_angle, wl.mask_angle, Ng)
        frac = wl.frac()
        rec = GradientRecon(wl.param, wl.angles, maskg, (Ng, Ng, Ng), fixed_frac=frac[Lg:],
                            tv_weight=1e-3, lr=1e-2, device=dev)
        Ig = rec.proj.project(torch.from_numpy(wl.conc).to(dev))
        Cg = torch.full((Lg, Ng, Ng, Ng), 0.5, device=dev)
        def once():
            rec.gradient(Cg, Ig)
    elif args.case == "xrf_adjoint_large":
        from fl_correction_b200 import phantoms
        from fl_correction_b200.xrf import XRFProjector
        wl = phantoms.make_workload(4)
        Nx, Lx, S = wl.N, len(wl.elements), args.case_slices
        sub = np.arange(4) * (len(wl.angles) // 4)
        maskx = generate_detector_mask(wl.mask_angle, wl.mask_angle, Nx)
        fr = wl.frac()[:, :S].copy()
        proj = XRFProjector(param_at_angles(wl.param, len(wl.angles), sub), wl.angles[sub], maskx,
                            (S, Nx, Nx), fixed_frac=fr[Lx:], device=dev)
        Cx = torch.from_numpy(fr[:Lx]).to(dev).contiguous()
        gx = torch.rand((Lx, len(sub), S, Nx), device=dev, generator=g)
        def once():
            proj.adjoint(Cx, gx)
    elif args.case == "bwd_large":
        # the row-band backward: 180 angles x --case-slices slices of 256^2
        N, A, B = 256, 180, args.case_slices
        atten = torch.rand((A, B, N, N), device=dev, generator=g)
        em = torch.full((A, 1), 0.02, device=dev)
        th = torch.linspace(0, math.pi, A + 1, device=dev)[:-1].contiguous()
        r = torch.rand((A, B, N), device=dev, generator=g)
        def once():
            AC.backward_emission_batch(atten, r, em, th)
    elif args.case in ("fwd", "bwd"):
        A, B = 120, args.case_slices
        atten = torch.rand((A, B, N, N), device=dev, generator=g)
        em = torch.full((A, 1), 0.02, device=dev)
        th = torch.linspace(0, math.pi, A + 1, device=dev)[:-1].contiguous()
        C = torch.rand((1, B, N, N), device=dev, generator=g)
        r = torch.rand((A, B, N), device=dev, generator=g)
        if args.case == "fwd":
            def once():
                AC.forward_emission_batch(atten, C, em, th)
        else:
            def once():
                AC.backward_emission_batch(atten, r, em, th)
    else:
        raise ValueError(args.case)
    for _ in range(args.warmup):
        once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    once()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "ms": round(e0.elapsed_time(e1), 4)}))


def main():
    args = parse()
    if args.case:
        run_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    device = torch.device("cuda", torch.cuda.current_device())
    if args.config in (2, 3, 4):
        if rank == 0:
            fn = run_batch if args.config == 3 else run_grad
            print(json.dumps(fn(args, device)), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    line = run_ours(args, rank, world, device)
    if rank == 0 and world == 1 and not args.no_parity:
        wl, mask, solver, I = build_problem(args.config, rank, device)
        line["parity"] = parity_leg(wl, mask, solver, I, device)
        del solver, I
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        import torch
        torch.cuda.empty_cache()
        line["reference_gpu_kernels"] = reference_gpu_leg(device)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, desc, cores, _ = cpu_sample(args.config)
        line["cpu_baseline"] = {"value": round(v, 6), "unit": "MLEM iters/s", "cores": cores,
                                "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
