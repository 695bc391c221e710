"""Golden vectors from the reference's own CUDA extension, run on a GPU.

The extension is compiled from the reference sources by oracle/build_ref.py
into oracle/_ref/ref_atten_cuda.so (its unmodified kernels, sm_100a).  This
script calls it through the reference's pybind API on seeded inputs and
writes inputs and outputs to tests/golden/ref_gpu.npz:

    python tests/golden/make_golden_refgpu.py [out.npz]

The reference kernels use global atomicAdd (forward_emission_batch,
backward_emission[_batch]) so their last bits vary between runs; the
fixtures record one run.
"""
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.build_ref import load_built  # noqa: E402


def main(out_path):
    ref = load_built()
    rng = np.random.default_rng(20240612)
    dev = "cuda"
    T = lambda x: torch.tensor(np.asarray(x), dtype=torch.float32, device=dev)
    out = {}
    # cone (atten_kernel) with a config-style mask and a general mask
    import fl_correction_b200.detector_mask as dm
    mask = dm.generate_detector_mask(13.309, 13.309, 20).astype(np.float32)
    mu = (rng.random((2, 9, 20, 20)) * 0.1).astype(np.float32)
    out["cone_mask"], out["cone_mu"] = mask, mu
    out["cone_out"] = ref.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    gmask = rng.random((5, 7, 3)).astype(np.float32)
    out["cone_gmask"] = gmask
    out["cone_gout"] = ref.cal_atten_cuda(T(mu), T(gmask)).cpu().numpy()
    # projector, batched and single slice
    A, B, R, H, W = 9, 3, 2, 24, 24
    atten = rng.random((A, B, H, W)).astype(np.float32)
    C = rng.random((R, B, H, W)).astype(np.float32)
    em = rng.uniform(0.5, 2.0, (A, R)).astype(np.float32)
    th = np.array([0.0, math.pi / 2, math.pi / 4, 1.0, 2.0, 3.0, -1.0, 0.3, 2.5], np.float32)
    ratio = rng.random((A, B, W)).astype(np.float32)
    out.update(p_atten=atten, p_C=C, p_em=em, p_theta=th, p_ratio=ratio)
    out["p_fwd_batch"] = ref.forward_emission_batch(T(atten), T(C), T(em), T(th)).cpu().numpy()
    out["p_bwd_batch"] = ref.backward_emission_batch(T(atten), T(ratio), T(em), T(th)).cpu().numpy()
    out["p_fwd"] = ref.forward_emission(T(atten[:, 0]), T(C[:, 0]), T(em), T(th)).cpu().numpy()
    out["p_bwd"] = ref.backward_emission(T(atten[:, 0]), T(ratio[:, 0]), T(em), T(th)).cpu().numpy()
    # MLEM, 20 iterations, with and without the Huber term
    I = out["p_fwd_batch"] * rng.uniform(0.8, 1.2, (A, B, W)).astype(np.float32)
    out["m_I"] = I
    C0 = np.ones((R, B, H, W), np.float32)
    out["m_beta"] = ref.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 20, 1e-3, 0.01).cpu().numpy()
    out["m_nobeta"] = ref.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 20, 0.0, 0.01).cpu().numpy()
    out["m_single"] = ref.mlem_cuda(T(C0[:, 0]), T(atten[:, 0]), T(em), T(th), T(I[:, 0]), 20).cpu().numpy()
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_gpu.npz"))
