"""Loader for the reference's own RPY kernels built by oracle/ref_build.py (test helper).

The libraries live in oracle/_ref/ and are built in the build container from
the reference sources; on a GPU machine they are used as shipped.
"""
import ctypes
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
REF_DIR = ROOT / "oracle" / "_ref"

_cache = {}


def variant_name(wall: bool, seg_dof: int) -> str:
    return f"{'wall' if wall else 'free'}{seg_dof}"


def available(variant: str) -> bool:
    return (REF_DIR / f"libref_rpy_{variant}.so").exists()


def load(variant: str):
    if variant not in _cache:
        L = ctypes.CDLL(str(REF_DIR / f"libref_rpy_{variant}.so"))
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.ref_set_sizes.argtypes = [i, i, i, i]
        L.ref_mss.argtypes = [vp, vp, vp, i, i]
        L.ref_mss_async.argtypes = [vp, vp, vp, i, i]
        L.ref_msb.argtypes = [vp, vp, vp, vp, i, i]
        L.ref_mbb.argtypes = [vp, vp, vp, i, i]
        L.ref_mbs.argtypes = [vp, vp, vp, vp, i, i]
        _cache[variant] = L
    return _cache[variant]


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def full_mobility(torch, variant, x_segs, f_segs, x_blobs=None, f_blobs=None):
    """The reference's evaluate_full_mobility (rpy_mobility_solver.cu:330-338) on one device.

    Host numpy arrays in the reference layouts in, numpy (v_segs [6N], v_blobs [3B]) out."""
    import numpy as np
    L = load(variant)
    dev = torch.device("cuda")
    xs = torch.as_tensor(np.asarray(x_segs, np.float32).ravel(), device=dev)
    fs = torch.as_tensor(np.asarray(f_segs, np.float32).ravel(), device=dev)
    ns = xs.numel() // 3
    nb = 0 if x_blobs is None else len(np.asarray(x_blobs).ravel()) // 3
    xb = torch.as_tensor(np.asarray(x_blobs if nb else np.zeros(3), np.float32).ravel(), device=dev)
    fb = torch.as_tensor(np.asarray(f_blobs if nb else np.zeros(3), np.float32).ravel(), device=dev)
    vs = torch.zeros(6 * max(ns, 1), device=dev)
    vb = torch.zeros(3 * max(nb, 1), device=dev)
    # NSWIM = 1, NFIL = ns (NSEG = 1) so that NSWIM*NFIL*NSEG = ns; NBLOB = nb.
    assert L.ref_set_sizes(1, 1, ns, nb) == 0
    assert L.ref_mss(ptr(vs), ptr(fs), ptr(xs), 0, ns) == 0
    if nb:
        assert L.ref_msb(ptr(vs), ptr(fb), ptr(xs), ptr(xb), 0, ns) == 0
        assert L.ref_mbb(ptr(vb), ptr(fb), ptr(xb), 0, nb) == 0
        if L.ref_prescribed():
            assert L.ref_mbs(ptr(vb), ptr(fs), ptr(xb), ptr(xs), 0, nb) == 0  # Mbs_mult accumulates
        else:
            vb2 = torch.zeros_like(vb)  # Mbs_mult overwrites when segments carry torques
            assert L.ref_mbs(ptr(vb2), ptr(fs), ptr(xb), ptr(xs), 0, nb) == 0
            torch.cuda.synchronize()
            vb += vb2
    torch.cuda.synchronize()
    return vs[:6 * ns].cpu().numpy(), vb[:3 * nb].cpu().numpy()
