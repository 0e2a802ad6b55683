"""The flow-field evaluator (cf_flow) against the reference's own flow_velocities kernel and the FP64 oracle.

The reference kernel (src/flow_field/flow_field_evaluator.cu) is built in FP64
by oracle/ref_build.py into oracle/_ref/libref_flow.so and launched as its
host code launches it.  The engine computes in FP32 with compensated sums;
tolerance 1e-5 relative L2, the mobility contract.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import flow as oflow
from cufcm_fil_b200 import _lib
from cufcm_fil_b200.flow import FlowFieldEvaluator

pytestmark = pytest.mark.gpu

REF_FLOW = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libref_flow.so"
TOL = 1e-5


def _ref_flow(torch, xf, xs, fs, xb, fb, xbod, ns_pb, nb_pb, mu, net):
    L = ctypes.CDLL(str(REF_FLOW))
    assert L.ref_flow_real_size() == 8
    vp = ctypes.c_void_p
    L.ref_flow_velocities.argtypes = [vp] * 7 + [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_int]
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64).ravel(), device="cuda")
    Xf, Xs, Fs, Xb, Fb, Xd = (d(a) for a in (xf, xs, fs, xb if xb is not None else np.zeros(3),
                                             fb if fb is not None else np.zeros(3), xbod))
    Vf = torch.zeros(xf.size, dtype=torch.float64, device="cuda")
    p = lambda t: vp(t.data_ptr())
    nbods = max(len(xs) // ns_pb, (len(xb) // nb_pb) if nb_pb else 0)
    rc = L.ref_flow_velocities(p(Vf), p(Xf), p(Fs), p(Fb), p(Xs), p(Xd), p(Xb), len(xf), ns_pb, nbods, nb_pb,
                               mu, int(net))
    assert rc == 0
    return Vf.cpu().numpy().reshape(-1, 3)


def _case(seed, n_bod, ns_pb, nb_pb, nf):
    rng = np.random.default_rng(seed)
    xbod = rng.uniform(-40, 40, (n_bod, 3)) + [0, 0, 60]
    xs = np.concatenate([c + rng.uniform(-10, 10, (ns_pb, 3)) for c in xbod])
    if nb_pb == 0:
        xs[:, 2] = np.abs(xs[:, 2] - 60) + 1.5   # half-space data: segments above the wall
    fs = rng.standard_normal((len(xs), 6))
    xb = fb = None
    if nb_pb:
        xb = np.concatenate([c + rng.uniform(-8, 8, (nb_pb, 3)) for c in xbod])
        fb = rng.standard_normal((len(xb), 3))
    xf = rng.uniform([-80, -80, 0.5], [80, 80, 120], (nf, 3))
    return xf, xs, fs, xb, fb, xbod


@pytest.mark.parametrize("n_bod,ns_pb,nb_pb,nf,net", [(1, 400, 0, 300, False), (1, 400, 0, 2000, True),
                                                       (3, 120, 90, 777, True), (2, 64, 50, 5, False)])
def test_flow_velocities_match_reference_kernel_and_oracle(cuda, n_bod, ns_pb, nb_pb, nf, net):
    xf, xs, fs, xb, fb, xbod = _case(nf + ns_pb, n_bod, ns_pb, nb_pb, nf)
    f32 = lambda a: None if a is None else np.asarray(a, np.float32).astype(np.float64)
    with FlowFieldEvaluator(nf, len(xs), 0 if xb is None else len(xb), n_bod, mu=1.0, remove_net_force=net) as ev:
        v = ev.velocities(xf, xs, fs, n_seg_per_body=ns_pb, x_blobs=xb, f_blobs=fb, n_blob_per_body=nb_pb,
                          x_bodies=xbod)
    v64 = oflow.flow_velocities(f32(xf), f32(xs), f32(fs), f32(xb), f32(fb), f32(xbod), n_seg_per_body=ns_pb,
                                n_blob_per_body=nb_pb, remove_net_force=net)
    assert oracle.rel_l2(v, v64) <= TOL
    if REF_FLOW.exists():
        vr = _ref_flow(cuda, f32(xf), f32(xs), f32(fs), f32(xb), f32(fb), f32(xbod), ns_pb, nb_pb, 1.0, net)
        assert oracle.rel_l2(vr, v64) <= 1e-12   # the reference kernel in FP64 is the oracle's formula
        assert oracle.rel_l2(v, vr) <= TOL


def test_flow_rejects_sizes_beyond_capacity(cuda):
    with FlowFieldEvaluator(10, 20) as ev:
        with pytest.raises(_lib.CufilError) as ei:
            ev.velocities(np.zeros((11, 3)), np.ones((20, 3)), np.zeros((20, 6)))
        assert ei.value.code == _lib.CF_EINVAL
        v = ev.velocities(np.zeros((0, 3)), np.ones((20, 3)), np.zeros((20, 6)))
        assert v.shape == (0, 3)
