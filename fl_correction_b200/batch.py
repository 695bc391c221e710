"""Batched corrected MLEM over several independent volumes of uneven size.

The reference reconstructs one volume at a time, and within a volume one
angle and one element at a time (FL/example/demo.py:244-336).  Here a list
of problems -- different sizes, element counts, angle counts, energies and
detector distances -- becomes one job:

* every problem gets its own device-resident `CorrectedMLEM` (attenuation,
  workspaces), built once;
* launch shapes are chosen per distinct problem shape by the project
  autotuner (`tune`), and set before that problem's launches are issued;
* the whole schedule of every problem -- attenuation rebuilt every k
  iterations, the MLEM iterations -- is captured once into a single CUDA
  graph, with the problems spread over several capture streams so that
  small volumes run side by side instead of leaving most SMs idle;
* `run()` replays that one graph.

`run_persistent()` is the other batched form: between attenuation rebuilds,
the MLEM iterations of every (volume, element) pair run as one
flc_mlem_multi_sizes call per iteration (one persistent launch per slice
width: clusters take (problem, slice) items of all volumes of that width
from a device work queue), optionally replayed as a CUDA graph of the whole
schedule (`capture_persistent`).

`run_loop()` is the plain single-volume path for comparison: the same
problems one after another, default launch shapes, no graph.
"""
import numpy as np
import torch

from . import _lib, tune
from .detector_mask import generate_detector_mask
from .recon import CorrectedMLEM

__all__ = ["BatchProblem", "BatchedMLEM", "assign_streams"]


class BatchProblem:
    """One volume of the batch: the param dict, angles (degrees), cone mask,
    shape (S, H, W), projections I (L, A, S, W) on the device, optional fixed
    fractions of the non-element compounds."""

    def __init__(self, param, angles_deg, mask, shape, I, fixed_frac=None, name=""):
        self.param, self.angles, self.mask = param, np.asarray(angles_deg, np.float64), mask
        self.shape, self.I, self.fixed_frac, self.name = tuple(shape), I, fixed_frac, name

    @property
    def work(self):
        """Relative cost: samples per MLEM iteration over all elements."""
        S, H, W = self.shape
        return len(self.param["elem_type"]) * len(self.angles) * S * H * W


def assign_streams(works, n_streams):
    """Greedy longest-first assignment of problems to streams (balanced total
    work per stream); returns a list of index lists."""
    order = sorted(range(len(works)), key=lambda i: -works[i])
    load = [0.0] * n_streams
    groups = [[] for _ in range(n_streams)]
    for i in order:
        j = min(range(n_streams), key=lambda k: load[k])
        groups[j].append(i)
        load[j] += works[i]
    return [g for g in groups if g]


class BatchedMLEM:
    """All problems' corrected MLEM (n_iter iterations, attenuation rebuilt
    every `recompute_every`) as one CUDA graph replay."""

    def __init__(self, problems, n_iter=20, recompute_every=5, n_streams=4, autotune=True,
                 device="cuda"):
        self.device = torch.device(device)
        self.problems = list(problems)
        self.n_iter, self.k = int(n_iter), int(recompute_every)
        self.solvers = [CorrectedMLEM(p.param, p.angles, p.mask, p.shape, fixed_frac=p.fixed_frac,
                                      device=self.device) for p in self.problems]
        self.C = [torch.ones((s.L,) + s.shape, dtype=torch.float32, device=self.device)
                  for s in self.solvers]
        self.I = [p.I.contiguous() for p in self.problems]
        self.groups = assign_streams([p.work for p in self.problems], max(1, int(n_streams)))
        self.knobs = [{} for _ in self.problems]
        if autotune:
            self._autotune()
        self.graph = None

    # -- launch shapes ------------------------------------------------------
    def _autotune(self):
        """proj.cluster for the fused MLEM iteration, per distinct (A, S, N)."""
        cache = {}
        for i, (p, s) in enumerate(zip(self.problems, self.solvers)):
            S, H, W = p.shape
            key = (len(p.angles), S, H)
            if key not in cache:
                best, _ = tune.tune_mlem(len(p.angles), S, H, W, self.device)["proj.cluster"]
                cache[key] = {"proj.cluster": best}
                tune.set_knob("proj.cluster", 0)
            self.knobs[i] = cache[key]

    def _issue(self, i):
        """Problem i's whole schedule on the current stream."""
        for name, v in self.knobs[i].items():
            tune.set_knob(name, v)
        try:
            C = self.C[i]
            C.fill_(1.0)
            self.solvers[i].run_into(C, self.I[i], self.n_iter, self.k)
        finally:
            for name in self.knobs[i]:
                tune.set_knob(name, 0)

    # -- the plain path -----------------------------------------------------
    def run_loop(self):
        """One problem after another on the current stream, default shapes."""
        for i, s in enumerate(self.solvers):
            C = self.C[i]
            C.fill_(1.0)
            s.run_into(C, self.I[i], self.n_iter, self.k)
        return self.C

    # -- the batched path ---------------------------------------------------
    def capture(self):
        """Record every problem's schedule into one CUDA graph (runs the
        schedule once eagerly first, so every launch plan is cached)."""
        streams = [torch.cuda.Stream(self.device) for _ in self.groups]
        cur = torch.cuda.current_stream(self.device)
        for j, g in enumerate(self.groups):           # warm-up with the same stream layout
            streams[j].wait_stream(cur)
            with torch.cuda.stream(streams[j]):
                for i in g:
                    self._issue(i)
        for s in streams:
            cur.wait_stream(s)
        torch.cuda.synchronize(self.device)
        self.graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(self.device)
        with torch.cuda.graph(self.graph, stream=cap):
            root = torch.cuda.current_stream(self.device)
            for s in streams:
                s.wait_stream(root)
            for j, g in enumerate(self.groups):
                with torch.cuda.stream(streams[j]):
                    for i in g:
                        self._issue(i)
            for s in streams:
                root.wait_stream(s)
        self._streams = streams
        return self.graph

    def run(self):
        """Replay the captured job (captures it on first use); returns the C list."""
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.C

    # -- the persistent multi-problem path -----------------------------------
    def _multi_args(self):
        Cs, ats, ems, ths, Is = [], [], [], [], []
        for s, C, I in zip(self.solvers, self.C, self.I):
            for l in range(s.L):
                Cs.append(C[l:l + 1])
                ats.append(s.atten[l])
                ems.append(s.em[l])
                ths.append(s.theta)
                Is.append(I[l])
        return Cs, ats, ems, ths, Is

    def _issue_persistent(self):
        betas = {(s.beta, s.delta) for s in self.solvers}
        if len(betas) != 1:
            raise ValueError("run_persistent: every volume must use the same beta and delta")
        beta, delta = betas.pop()
        for C in self.C:
            C.fill_(1.0)
        args = self._multi_args()
        done = 0
        while done < self.n_iter:
            kk = min(self.k, self.n_iter - done)
            for s, C in zip(self.solvers, self.C):
                s.recompute_attenuation(C)
            self._ws_multi = _lib.mlem_multi(*args, kk, beta, delta, getattr(self, "_ws_multi", None))
            done += kk

    def run_persistent(self):
        """The schedule with one persistent MLEM launch per iteration for all
        (volume, element) problems; replays the captured graph when
        `capture_persistent` has run.  Returns the C list."""
        if getattr(self, "graph_persistent", None) is not None:
            self.graph_persistent.replay()
        else:
            self._issue_persistent()
        return self.C

    def capture_persistent(self):
        """Record the persistent schedule into one CUDA graph (one eager run
        first, so that the workspace and every launch plan exist)."""
        self._issue_persistent()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=torch.cuda.Stream(self.device)):
            self._issue_persistent()
        self.graph_persistent = g
        return g


def problems_from_workloads(workloads, device="cuda"):
    """BatchProblems from `phantoms.Workload`s: the projections are made on the
    device from each truth through that volume's own attenuation."""
    out = []
    for wl in workloads:
        N = wl.N
        mask = generate_detector_mask(wl.mask_angle, wl.mask_angle, N)
        L = len(wl.elements)
        frac = wl.frac()
        s = CorrectedMLEM(wl.param, wl.angles, mask, (N, N, N), fixed_frac=frac[L:], device=device)
        truth = torch.from_numpy(wl.conc).to(device)
        s.recompute_attenuation(truth)
        I = s.project(truth).contiguous()
        del s
        out.append(BatchProblem(wl.param, wl.angles, mask, (N, N, N), I, fixed_frac=frac[L:],
                                name=wl.name))
    return out
