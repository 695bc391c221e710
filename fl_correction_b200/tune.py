"""Launch-shape autotuner for the native kernels.

The library picks launch shapes from the device's SM count and shared
memory; this module times the alternatives on the actual problem shape with
CUDA events and keeps the fastest through ``flc_tune_set``:

  proj.cluster   CTAs per slice cluster of the backward projector / fused
                 MLEM kernel (1, 2, 4, 8)
  proj.apc       angles per CTA of the forward projector
  cone.variant   TMA 16x8 tile, TMA 8x4 tile, the plain separable kernel or
                 the spectral form (FFTs of the depth planes)
  atten.chunk    angles per attenuation-pipeline pass
  proj.bwd       backward: splat with shared atomics, splat in nine disjoint
                 phases, gather per pixel, or splat by column segments

Every candidate is checked against the automatic choice before it is timed
(the results must agree to FP32 round-off), so tuning never changes answers
beyond the summation order.  ``python -m fl_correction_b200.tune`` prints the
table for the benchmark shapes.
"""
import json
import math
import sys

import torch

from . import _lib

__all__ = ["set_knob", "get_knob", "knobs", "time_ms", "tune_projector", "tune_cone",
           "tune_mlem", "autotune"]

KNOBS = ("proj.cluster", "proj.apc", "cone.variant", "atten.chunk", "proj.bwd")


def set_knob(name, value):
    _lib.call("flc_tune_set", name.encode(), int(value))


def get_knob(name):
    v = _lib.query("flc_tune_get", name.encode())
    if v < 0:
        raise KeyError(name)
    return v


def knobs():
    return {k: get_knob(k) for k in KNOBS}


def time_ms(fn, warmup=2, reps=5):
    """Median CUDA-event time of fn() on the current stream (ms)."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ts.sort()
    return ts[len(ts) // 2]


def _sweep(name, values, run, check=None):
    """Time run() for each knob value; keep the fastest that passes check."""
    old = get_knob(name)
    ref = run() if check is not None else None
    table = []
    try:
        for v in values:
            set_knob(name, v)
            if check is not None and not check(ref, run()):
                table.append((v, None))
                continue
            table.append((v, time_ms(run)))
    finally:
        set_knob(name, old)
    ok = [(t, v) for v, t in table if t is not None]
    best = min(ok)[1] if ok else old
    set_knob(name, best)
    return best, table


def _close(a, b, tol=1e-4):
    return float((a - b).abs().max()) <= tol * max(float(b.abs().max()), 1e-30)


def _proj_inputs(A, B, H, W, dev, seed=0):
    g = torch.Generator(device=dev).manual_seed(seed)
    atten = torch.rand((A, B, H, W), device=dev, generator=g)
    em = torch.full((A, 1), 0.02, device=dev)
    th = torch.linspace(0, math.pi, A + 1, device=dev)[:-1].contiguous()
    C = torch.rand((1, B, H, W), device=dev, generator=g)
    r = torch.rand((A, B, W), device=dev, generator=g)
    return atten, em, th, C, r


def tune_projector(A, B, H, W, device="cuda"):
    """proj.bwd and proj.cluster for the backward projector, proj.apc for the
    forward."""
    from .cuda_lib import atten_cuda as AC
    dev = torch.device(device)
    atten, em, th, C, r = _proj_inputs(A, B, H, W, dev)
    bwd = lambda: AC.backward_emission_batch(atten, r, em, th)  # noqa: E731
    fwd = lambda: AC.forward_emission_batch(atten, C, em, th)  # noqa: E731
    out = {}
    out["proj.bwd"] = _sweep("proj.bwd", [0, 1, 2, 3, 4], bwd, _close)
    out["proj.cluster"] = _sweep("proj.cluster", [0, 1, 2, 4, 8], bwd, _close)
    apcs = sorted({0} | {a for a in (1, 2, 3, 4, 6, 8, 12, 16) if a <= A})
    out["proj.apc"] = _sweep("proj.apc", apcs, fwd, _close)
    return out


def tune_mlem(A, B, H, W, device="cuda"):
    """proj.cluster for the fused MLEM iteration (shares the knob with the
    backward projector: call after tune_projector to give MLEM the last word)."""
    from .cuda_lib import atten_cuda as AC
    dev = torch.device(device)
    atten, em, th, C, _ = _proj_inputs(A, B, H, W, dev)
    I = AC.forward_emission_batch(atten, C * 0.7, em, th)
    run = lambda: AC.mlem_cuda_batch(C, atten, em, th, I, 2)  # noqa: E731
    return {"proj.cluster": _sweep("proj.cluster", [0, 1, 2, 4, 8], run, _close)}


def tune_cone(n_a, L, N, A, mask, device="cuda"):
    """cone.variant for one attenuation-pipeline chunk of n_a angles x L lines."""
    from .detector_mask import factor_mask
    dev = torch.device(device)
    u, v = (torch.from_numpy(x).to(dev) for x in factor_mask(mask))
    g = torch.Generator(device=dev).manual_seed(0)
    mu = torch.rand((n_a, L, N, N, N), device=dev, generator=g) * 0.01
    atten = torch.ones((L, A, N, N, N), device=dev)
    nb = int(_lib.query("flc_cone_fft_workspace_bytes", n_a * L, N, N, N, *mask.shape))
    ws = _lib.workspace(nb, dev) if nb else None

    def run():
        atten.fill_(1.0)
        _lib.call("flc_cone_atten_apply_ws", _lib.ptr(mu), _lib.ptr(u), _lib.ptr(v),
                  _lib.ptr(atten), n_a, L, N, N, N, A, 0, *mask.shape, _lib.ptr(ws), nb,
                  _lib.stream())
        return atten[:, :n_a].clone()

    return {"cone.variant": _sweep("cone.variant", [0, 1, 2, 3, 4], run, _close)}


def autotune(A, S, N, L, mask, chunk, device="cuda"):
    """Tune every knob for an (L elements, A angles, S x N x N) problem; returns
    {knob: (chosen value, [(candidate, ms or None if rejected), ...])}."""
    res = {}
    res.update(tune_projector(A, S, N, N, device))
    res.update(tune_cone(max(1, chunk), L, N, A, mask, device))
    res.update(tune_mlem(A, S, N, N, device))
    return res


def main(argv=None):
    import argparse
    from .detector_mask import generate_detector_mask
    p = argparse.ArgumentParser(description="time the launch-shape alternatives")
    p.add_argument("--angles", type=int, default=120)
    p.add_argument("--slices", type=int, default=16)
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--lines", type=int, default=3)
    p.add_argument("--chunk", type=int, default=2)
    a = p.parse_args(argv)
    mask = generate_detector_mask(13.309, 13.309, a.n)
    res = autotune(a.angles, a.slices, a.n, a.lines, mask, a.chunk)
    for k, (best, table) in res.items():
        print(json.dumps({"knob": k, "best": best,
                          "ms": {str(v): (None if t is None else round(t, 4)) for v, t in table}}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
