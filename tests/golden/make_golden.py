"""Generate golden vectors from the reference's own Python code (CPU).

Run here, where the reference checkout is readable:
    python tests/golden/make_golden.py            # writes tests/golden/ref_cpu.npz

The reference package cannot be imported as-is (its ``__init__`` pulls in
xraylib / scikit-image / h5py / matplotlib, none installed), so the modules
on the hot path are imported one by one with permissive stub modules standing
in for those libraries and for the CUDA extension.  Nothing of the stubbed
libraries is reached by the functions called below.

The only reference piece that needs a GPU is ``cal_atten_cuda`` inside
``torch_xrf_atten_3D``; for the composite golden it is replaced by an
independent FP64 torch formulation of the same correlation (a ``conv3d`` with
the mask), which the GPU goldens of ``make_golden_refgpu.py`` pin against the
reference kernel itself.
"""
import importlib.abc
import importlib.machinery
import json
import math
import os
import sys
import types
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.build_ref import ref_root  # noqa: E402

REF = ref_root(required=True)
STUBBED = ("xraylib", "skimage", "matplotlib", "h5py", "pystackreg", "bm3d",
           "tomopy", "pyxas", "porespy")
CUDA_NAMES = ("cal_atten_cuda", "forward_emission", "backward_emission",
              "forward_emission_batch", "backward_emission_batch", "mlem_cuda",
              "mlem_cuda_batch")


class _Any(types.ModuleType):
    def __getattr__(self, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return _Any(self.__name__ + "." + k)

    def __call__(self, *a, **k):
        return None


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in STUBBED:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _Any(spec.name)
        m.__path__ = []
        return m

    def exec_module(self, m):
        pass


def import_reference():
    """Make FL.<hot-path modules> importable from the reference checkout."""
    if "FL.torch_functions" in sys.modules:
        return
    sys.meta_path.insert(0, _StubFinder())
    fl = os.path.join(REF, "FL")
    pkg = types.ModuleType("FL")
    pkg.__path__ = [fl]
    sys.modules["FL"] = pkg
    cl = types.ModuleType("FL.cuda_lib")
    cl.__path__ = [os.path.join(fl, "cuda_lib")]
    sys.modules["FL.cuda_lib"] = cl
    ac = types.ModuleType("FL.cuda_lib.atten_cuda")
    for n in CUDA_NAMES:
        setattr(ac, n, None)
    sys.modules["FL.cuda_lib.atten_cuda"] = ac


def cone_conv3d(mu, mask):
    """Independent FP64 statement of atten_kernel (atten_cuda_kernel.cu:10-57)
    as a zero-padded 3-D correlation: out[k,z,x,y] = sum mask[dz,dx,dy] *
    mu[k, z+dz-Mz//2, x+dx, y+dy-My//2]."""
    import torch
    import torch.nn.functional as F
    mu = torch.as_tensor(mu, dtype=torch.float64)
    m = torch.as_tensor(np.asarray(mask), dtype=torch.float64)
    Mz, Mx, My = m.shape
    K, Z, X, Y = mu.shape
    hz, hy = Mz // 2, My // 2
    # pad so that index z+dz-hz, x+dx, y+dy-hy is in range for every tap
    p = F.pad(mu[:, None], (hy, My - 1 - hy, 0, Mx - 1, hz, Mz - 1 - hz))
    out = F.conv3d(p, m[None, None])
    return out[:, 0, :Z, :X, :Y]


def make_param(n_ch, rng, energy_len=None):
    elems = ["Fe", "Ni", "Cu", "Zn"][:n_ch]
    comps = ["Fe2O3", "NiO", "CuO", "ZnO"][:n_ch]
    cs = {"elem_type": elems, "elem_compound": comps}
    for c in comps:
        v = rng.uniform(20.0, 200.0, size=energy_len or 1)
        cs[f"{c}-x"] = v
        for e in elems:
            cs[f"{c}-{e}"] = float(rng.uniform(20.0, 300.0))
    rho = {c: float(rng.uniform(3.0, 8.0)) for c in comps}
    em = {e: rng.uniform(0.5, 2.0, size=energy_len or 1) for e in elems}
    return {"cs": cs, "rho": rho, "pix": 1e-4, "elem_type": elems,
            "elem_compound": comps, "em_cs": em}


def main():
    import torch
    import_reference()
    warnings.filterwarnings("ignore")
    import FL.torch_image_util as tiu
    import FL.torch_functions as tf
    import FL.detector_mask as dm
    import FL.atten_util as au

    rng = np.random.default_rng(20240611)
    out = {}
    meta = {}

    # ---- rotation (FL/torch_image_util.py:13-114) ------------------------
    rot_x = rng.random((2, 3, 20, 20)).astype(np.float32)
    rot_x[:, :, 5:9, 3:16] += 2.0
    angles = np.array([0.0, 0.37, 1.2, math.pi / 2, 2.9, -0.8])
    out["rot_x"] = rot_x
    out["rot_theta"] = angles
    for i, th in enumerate(angles):
        # the reference passes a float64 0-d tensor (FL/core.py:35,43)
        y = tiu.torch_rotate_image_nd(torch.tensor(rot_x), torch.tensor(th, dtype=torch.float64))
        out[f"rot_y{i}"] = y.numpy()
    rot_x3 = rng.random((2, 17, 23)).astype(np.float32)       # (C,H,W), H != W
    out["rot_hw_x"] = rot_x3
    out["rot_hw_y"] = tiu.torch_rotate_image_nd(torch.tensor(rot_x3), 0.61).numpy()

    # ---- rot90 (FL/torch_image_util.py:117-155) -------------------------
    r90 = rng.random((2, 3, 7, 7)).astype(np.float32)
    out["r90_x"] = r90
    out["r90_clock"] = tiu.torch_rot90_4D(torch.tensor(r90), ax=0, mode="clock").numpy()
    out["r90_cclock"] = tiu.torch_rot90_4D(torch.tensor(r90), ax=0, mode="c-clock").numpy()

    # ---- detector mask (FL/detector_mask.py:22-106) ---------------------
    mask_cases = [(13.309, 13.309, 16), (13.309, 13.309, 20), (13.309, 13.309, 32),
                  (13.309, 13.309, 64), (10.0, 20.0, 24), (15.0, 60.0, 12)]
    meta["mask_cases"] = mask_cases
    for i, (a, b, L) in enumerate(mask_cases):
        out[f"mask{i}"] = dm.generate_detector_mask(a, b, L)

    # ---- per-angle parameter selection (FL/atten_util.py:63-135) --------
    n_angle = 5
    param = make_param(3, rng, energy_len=n_angle)
    meta["param"] = {"cs": {k: (v.tolist() if isinstance(v, np.ndarray) else v)
                            for k, v in param["cs"].items()},
                     "rho": param["rho"], "pix": param["pix"],
                     "elem_type": param["elem_type"], "elem_compound": param["elem_compound"],
                     "em_cs": {k: v.tolist() for k, v in param["em_cs"].items()}}
    sel = []
    for a in range(n_angle):
        p = au.extract_single_value_param(param, a)
        sel.append({"cs": {k: (np.asarray(v).tolist() if not isinstance(v, str) and k not in
                               ("elem_type", "elem_compound") else v)
                           for k, v in p["cs"].items()},
                    "em_cs": {k: np.asarray(v).tolist() for k, v in p["em_cs"].items()}})
    meta["param_selected"] = sel
    meta["em_cs_elem_Ni"] = np.asarray(au.extract_em_cs_elem(param, "Ni")).tolist()

    # ---- attenuation maps (FL/torch_functions.py:8-176) -----------------
    n_ch, S, N = 3, 6, 16
    frac = (rng.random((n_ch, S, N, N)) * 0.8).astype(np.float32)
    frac[:, :, 4:10, 6:12] += 0.5
    out["atten_frac"] = frac
    p1 = au.extract_single_value_param(param, 2)
    # scale cross sections so mu*pix*N ~ O(1)
    p1["pix"] = 2e-3
    meta["atten_param"] = {"cs": {k: (np.asarray(v).tolist() if k not in
                                      ("elem_type", "elem_compound") else v)
                                  for k, v in p1["cs"].items()},
                           "rho": p1["rho"], "pix": p1["pix"]}
    ft = torch.tensor(frac)
    out["mu_x"] = tf.torch_extract_3D_mu_xray(ft, p1).numpy()
    out["mu_xrf"] = tf.torch_extract_3D_mu_xrf(ft, p1).numpy()
    out["atten_x"] = tf.torch_xray_atten_3D(ft, p1)
    mask = dm.generate_detector_mask(13.309, 13.309, N)
    out["xrf_mask"] = mask
    # the reference calls cal_atten_cuda on CUDA tensors; stand in with the
    # FP64 correlation above, returning the same FP32 tensor type
    tf.cal_atten_cuda = lambda mu, m: cone_conv3d(mu, m.cpu().numpy()).to(torch.float32)
    tf.torch.cuda.synchronize = lambda *a, **k: None
    out["atten_xrf_r"] = tf.torch_xrf_atten_3D(ft, p1, mask, position_det="r")
    out["atten_xrf_l"] = tf.torch_xrf_atten_3D(ft, p1, mask, position_det="l")
    # rotated-then-attenuated, as FL/core.py:43-45,75-79 do per angle
    th = 0.7
    fr = tiu.torch_rotate_image_nd(ft, torch.tensor(th, dtype=torch.float64))
    out["pipe_theta"] = np.array(th)
    out["pipe_atten_x"] = tf.torch_xray_atten_3D(fr, p1)
    out["pipe_atten_xrf"] = tf.torch_xrf_atten_3D(fr, p1, mask)
    # the direct correlation itself, for the oracle's cone restatement
    mu_c = rng.random((2, 5, 16, 12)).astype(np.float32)
    out["cone_mu"] = mu_c
    out["cone_out"] = cone_conv3d(mu_c, mask).numpy()

    # ---- reference-spectrum incident cross section (XANES) ---------------
    # FL/torch_functions.py:22-37 -> FL/cross_section_util.py:44-66, which
    # calls cal_frac without importing it: the FL.core function it names is
    # put into that module's namespace.  skimage is stubbed, so cal_frac's
    # Otsu mask falls back to 1 (FL/core.py:177-179).
    import FL.core as core
    import FL.cross_section_util as csu
    csu.cal_frac = core.cal_frac
    rng2 = np.random.default_rng(20240612)
    n_angle = 5
    pr = make_param(3, rng2, energy_len=n_angle)
    comps = pr["elem_compound"]
    ref_comp = comps[1]
    pr["cs"]["n_ref"] = 2
    for i in range(2):
        pr["cs"][f"{ref_comp}-x_ref{i + 1}"] = rng2.uniform(30.0, 160.0, n_angle)
    pr["pix"] = 8e-4
    fr = (rng2.random((3, 6, 16, 16)) * 0.8).astype(np.float32)
    fr[:, :, 3:11, 5:12] += 0.4
    ref3 = rng2.uniform(0.1, 1.0, (2, 6, 16, 16)).astype(np.float32)
    ref3[0, :, 2:8, 4:14] *= 4.0
    out["xref_frac"] = fr
    out["xref_ref3d"] = ref3
    a_id = 3
    ang = np.linspace(0.0, 180.0, n_angle, endpoint=False)
    meta["xref"] = {"ref_comp": ref_comp, "angle_id": a_id, "angles_deg": ang.tolist(),
                    "param": {"cs": {k: (np.asarray(v).tolist() if k not in
                                         ("elem_type", "elem_compound") else v)
                                     for k, v in pr["cs"].items()},
                              "rho": pr["rho"], "pix": pr["pix"], "elem_type": pr["elem_type"],
                              "elem_compound": pr["elem_compound"],
                              "em_cs": {k: np.asarray(v).tolist() for k, v in pr["em_cs"].items()}}}
    d_ref = {"use_ref": True, "ref_3D": ref3, "ref_comp": ref_comp}
    d_rot = au.update_dict_use_ref_at_angle(d_ref, ang[a_id])
    p_a = au.extract_single_value_param(pr, a_id, d_rot)
    fr_rot = tiu.torch_rotate_image_nd(torch.tensor(fr), torch.tensor(ang[a_id] / 180.0 * np.pi,
                                                                      dtype=torch.float64))
    out["xref_atten_x"] = tf.torch_xray_atten_3D(fr_rot, p_a, d_rot)
    out["xref_ref3d_rot"] = np.asarray(d_rot["ref_3D"], np.float32)
    out["xref_mu_x"] = tf.torch_extract_3D_mu_xray(fr_rot, p_a, d_rot).numpy()
    meta["xref"]["selected_x_ref"] = [float(p_a["cs"][f"{ref_comp}-x_ref{i + 1}"]) for i in range(2)]

    # ---- cal_frac (FL/core.py:159-205) -----------------------------------
    # skimage is stubbed, so adaptive_threshold fails and cal_frac falls back
    # to mask = 1 (FL/core.py:177-179), the case flc_cal_frac reproduces
    rng3 = np.random.default_rng(20240613)
    cimg = (rng3.random((3, 6, 20, 20)) * 1.5).astype(np.float32)
    cimg[:, :, :3, :] = 0.0                    # empty rows: zero sums
    cimg[1, 2:4, 5:9, 5:9] = -0.2              # negatives (rm_abnormal)
    cimg[2, :, 10:, 12:] *= 6.0                # a bright corner for the clamps
    out["calfrac_img"] = cimg
    r = core.cal_frac(cimg, scale_range=[0.02, 0.98], enable_scale=True, scale_limit=0.95)
    out["calfrac_default"] = r["frac"]
    out["calfrac_default_sum"] = r["img_sum"]
    meta["calfrac_pix_max"] = float(r["pix_max"])
    r = core.cal_frac(cimg, scale_range=[], enable_scale=False)
    out["calfrac_plain"] = r["frac"]
    r = core.cal_frac(cimg, scale_range=[0.1, 0.7], enable_scale=True, scale_limit=0.5)
    out["calfrac_other"] = r["frac"]

    # ---- torch_2D_xray_atten_with_ref[_vectorize] (FL/torch_functions.py:181,247)
    # a non-square slice (the aspect terms of both rotations), negative
    # entries (the relu of the vectorised form) and mu above 1 (the floors)
    import torch
    rng4 = np.random.default_rng(20240614)
    H2, W2, n_ref2 = 20, 26, 3
    xc = rng4.random((n_ref2, H2, W2)).astype(np.float32)
    xc[1, 4:7, 3:9] = -0.6
    xo = (rng4.random((H2, W2)) * 0.5).astype(np.float32)
    xth = np.array([0.0, 0.4, 1.3, 2.5, -0.7], np.float32)
    xcs = (rng4.random((len(xth), n_ref2)) * 3.0).astype(np.float32)
    xcs[2, 0] = 60.0                           # one angle past the floors
    xrho = (1.0 + rng4.random((H2, W2)) * 4.0).astype(np.float32)
    xpix = 0.05
    for k, v in (("C", xc), ("C_other", xo), ("theta", xth), ("cs_ref", xcs), ("rho", xrho)):
        out["xray2d_" + k] = v
    meta["xray2d_pix"] = xpix
    targs = [torch.from_numpy(a) for a in (xc, xo, xth, xcs, xrho)] + [xpix]
    out["xray2d_out"] = tf.torch_2D_xray_atten_with_ref(*targs).numpy()
    out["xray2d_vec_out"] = tf.torch_2D_xray_atten_with_ref_vectorize(*targs).numpy()

    np.savez_compressed(os.path.join(HERE, "ref_cpu.npz"), **out)
    with open(os.path.join(HERE, "ref_cpu.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", os.path.join(HERE, "ref_cpu.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
