"""Batched corrected MLEM (several uneven volumes, one CUDA graph) against the
plain per-volume loop and against a single-volume CorrectedMLEM run."""
import numpy as np
import pytest
import torch

from fl_correction_b200 import phantoms
from fl_correction_b200.batch import BatchedMLEM, problems_from_workloads
from fl_correction_b200.recon import CorrectedMLEM
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def test_graph_replay_matches_the_plain_loop():
    ws = phantoms.make_batch_workloads(5, sizes=(24, 32, 40), n_iter=6, recompute_every=3)
    probs = problems_from_workloads(ws)
    b = BatchedMLEM(probs, n_iter=6, recompute_every=3, n_streams=3, autotune=True)
    loop = [c.clone() for c in b.run_loop()]
    torch.cuda.synchronize()
    out = [c.clone() for c in b.run()]
    out2 = [c.clone() for c in b.run()]            # a second replay gives the same job
    torch.cuda.synchronize()
    for a, c, d in zip(loop, out, out2):
        assert rel_err(c.cpu().numpy(), a.cpu().numpy()) < 1e-5
        assert rel_err(d.cpu().numpy(), a.cpu().numpy()) < 1e-5
    # and the loop equals a stand-alone solver on the first problem
    p = probs[0]
    s = CorrectedMLEM(p.param, p.angles, p.mask, p.shape, fixed_frac=p.fixed_frac)
    ref = s.run(p.I, n_iter=6, recompute_every=3)
    assert rel_err(loop[0].cpu().numpy(), ref.cpu().numpy()) < 1e-5


def test_persistent_form_matches_the_plain_loop():
    """run_persistent: one persistent launch per MLEM iteration for every
    (volume, element) problem of uneven sizes, eager and replayed as a graph,
    against the plain loop."""
    ws = phantoms.make_batch_workloads(4, sizes=(24, 32, 40), n_iter=6, recompute_every=3)
    probs = problems_from_workloads(ws)
    b = BatchedMLEM(probs, n_iter=6, recompute_every=3, n_streams=2, autotune=False)
    loop = [c.clone() for c in b.run_loop()]
    eager = [c.clone() for c in b.run_persistent()]
    b.capture_persistent()
    replay = [c.clone() for c in b.run_persistent()]
    torch.cuda.synchronize()
    for a, e, r in zip(loop, eager, replay):
        assert rel_err(e.cpu().numpy(), a.cpu().numpy()) < 1e-5
        assert rel_err(r.cpu().numpy(), a.cpu().numpy()) < 1e-5
