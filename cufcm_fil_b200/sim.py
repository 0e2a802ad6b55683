"""Host mirror of the reference's mobility-solver generic layer for prescribed cilia on a wall.

``WallCiliaSimulation`` stands in for the pair (swimmer/filament objects,
``mobility_solver``) that ``cilia_sim_main.cu`` drives for CILIA_TYPE 3 on an
INFINITE_PLANE_WALL: one :meth:`step` is filament::initial_guess followed by
mobility_solver::compute_velocities (cilia_sim_main.cu:405-416), executed on
the device by libcufil.so.  The component methods keep the reference's names
(``initial_guess``, ``assemble_rhs``, ``apply_preconditioner_new``,
``system_matrix_mult_new``) so that a caller can test or drive each stage.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


@dataclass
class GmresResult:
    iterations: int
    relative_residual: float
    status: int


def _sim_config(keep: list, *, bases, nseg=20, seg_sep=2.6, beat=_lib.CF_BEAT_FULFORD_BLAKE, dt=1.0 / 300,
                dynamic_phase=True, dynamic_angle=True, spring_factor=0.01, gmres_tol=1e-6, gmres_max_iter=350,
                precond=_lib.CF_PRECOND_BLOCK_DIAG, omega0=None, phase0=None, angle0=None, phase_refs=None,
                angle_refs=None, s_table=None, s_tol_factor=0.0, device=0, line_patch=0, precond_refresh=0):
    """cf_sim_config of one array; the arrays it points to are appended to `keep` (kept alive by the caller)."""
    bases = np.ascontiguousarray(bases, np.float64).reshape(-1, 3)
    keep.append(bases)
    f = bases.shape[0]

    def arr(x, n=None):
        if x is None:
            return None
        a = np.ascontiguousarray(x, np.float64).ravel()
        if n is not None:
            assert a.size == n, (a.size, n)
        keep.append(a)
        return a

    om, ph, an = arr(omega0, f), arr(phase0, f), arr(angle0, f)
    pr, ar = arr(phase_refs), arr(angle_refs)
    st = None if s_table is None else np.ascontiguousarray(s_table, np.float64)
    if st is not None:
        keep.append(st)
    return _lib.SimConfig(
        n_fil=f, n_seg=int(nseg), seg_sep=float(seg_sep), beat=int(beat), dynamic_phase=int(bool(dynamic_phase)),
        dynamic_angle=int(bool(dynamic_angle)), dt=float(dt), spring_factor=float(spring_factor),
        gmres_tol=float(gmres_tol), gmres_max_iter=int(gmres_max_iter), precond=int(precond),
        base_pos=_p(bases), omega0=_p(om), phase0=_p(ph), angle0=_p(an),
        gen_phase_force_refs=_p(pr), n_gen_phase_refs=0 if pr is None else pr.size,
        gen_angle_force_refs=_p(ar), n_gen_angle_refs=0 if ar is None else ar.size,
        s_values_ref=_p(st), s_ref_rows=0 if st is None else st.shape[0],
        s_ref_cols=0 if st is None else st.shape[1], s_tol_factor=float(s_tol_factor), device=int(device),
        line_patch=int(line_patch), precond_refresh=int(precond_refresh))


class WallCiliaSimulation:
    def __init__(self, *, bases, nseg=20, **kw):
        self.bases = np.ascontiguousarray(bases, np.float64).reshape(-1, 3)
        self.n_fil = self.bases.shape[0]
        self.nseg = int(nseg)
        self._keep = []
        cfg = _sim_config(self._keep, bases=self.bases, nseg=nseg, **kw)
        h = ctypes.c_void_p()
        _lib.call("cf_sim_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        self.size = _lib.load().cf_sim_system_size(h)
        self.n_seg_total = self.n_fil * self.nseg

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_sim_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- whole step -------------------------------------------------------
    def step(self, nt: int) -> GmresResult:
        """filament::initial_guess + mobility_solver::compute_velocities for step nt (synchronous)."""
        it = ctypes.c_int()
        rel = ctypes.c_double()
        rc = _lib.call("cf_sim_step", self._h, int(nt), ctypes.byref(it), ctypes.byref(rel),
                       ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED))
        return GmresResult(it.value, rel.value, rc)

    def step_io(self, nt: int, state_in=None, state_out=None, x_segs=None, f_segs=None) -> GmresResult:
        """One step with its host traffic in one call: `state_in` / `state_out` are (phase, angle, phase_dot,
        angle_dot) float64 host arrays (numpy or pinned torch; None skips), x_segs [3N] / f_segs [6N] float32."""
        def q(a):
            if a is None:
                return None
            return ctypes.c_void_p(a.ctypes.data if hasattr(a, "ctypes") else a.data_ptr())
        si = list(state_in) if state_in is not None else [None] * 4
        so = list(state_out) if state_out is not None else [None] * 4
        it = ctypes.c_int()
        rel = ctypes.c_double()
        rc = _lib.call("cf_sim_step_io", self._h, int(nt), *(q(a) for a in si), *(q(a) for a in so), q(x_segs),
                       q(f_segs), ctypes.byref(it), ctypes.byref(rel), ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED))
        return GmresResult(it.value, rel.value, rc)

    def step_async(self, nt: int):
        """Enqueues step nt (one graph launch); read the solve with :meth:`last_solve`."""
        _lib.call("cf_sim_step_async", self._h, int(nt))

    def last_solve(self) -> GmresResult:
        it = ctypes.c_int()
        rel = ctypes.c_double()
        rc = _lib.call("cf_sim_last_solve", self._h, ctypes.byref(it), ctypes.byref(rel),
                       ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED))
        return GmresResult(it.value, rel.value, rc)

    # -- stages -----------------------------------------------------------
    def initial_guess(self, nt: int):
        _lib.call("cf_sim_initial_guess", self._h, int(nt))

    def assemble_rhs(self, nt: int = 0) -> np.ndarray:
        out = np.zeros(self.size)
        _lib.call("cf_sim_assemble_rhs", self._h, int(nt), _p(out))
        return out

    def apply_preconditioner_new(self, v) -> np.ndarray:
        v = np.ascontiguousarray(v, np.float64)
        out = np.zeros(self.size)
        _lib.call("cf_sim_apply_preconditioner", self._h, _p(v), _p(out))
        return out

    def system_matrix_mult_new(self, v) -> np.ndarray:
        v = np.ascontiguousarray(v, np.float64)
        out = np.zeros(self.size)
        _lib.call("cf_sim_system_matvec", self._h, _p(v), _p(out))
        return out

    def write_data(self, save_step: int, period: float, prefix: str) -> None:
        """Appends the reference's data files <prefix>_{seg_states,body_states,true_states,seg_vels,seg_forces}.dat
        (cf_sim_write_data)."""
        _lib.call("cf_sim_write_data", self._h, int(save_step), float(period), str(prefix).encode())

    def write_config(self, prefix: str, total_steps: int) -> None:
        """<prefix>_fil_references.dat and <prefix>.par (cf_sim_write_config)."""
        _lib.call("cf_sim_write_config", self._h, str(prefix).encode(), int(total_steps))

    def solve_linear_system(self, rhs, x0=None, tol: float = 1e-6, max_iter: int = 350):
        """GMRES on a given RHS for the current geometry (cf_sim_solve); returns (x, GmresResult).
        The solution becomes the next step's warm start and its rate rows the filament rates."""
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.zeros(self.size) if x0 is None else np.array(x0, np.float64)
        it, rel = ctypes.c_int(), ctypes.c_double()
        rc = _lib.call("cf_sim_solve", self._h, _p(rhs), _p(x), float(tol), int(max_iter), ctypes.byref(it),
                       ctypes.byref(rel), ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED, _lib.CF_NONFINITE))
        return x, GmresResult(it.value, rel.value, rc)

    # -- state ------------------------------------------------------------
    def stream_handle(self) -> int:
        """cudaStream_t of the engine's stream (for events / external streams)."""
        h = ctypes.c_void_p()
        _lib.call("cf_sim_stream", self._h, ctypes.byref(h))
        return h.value or 0

    def set_state(self, phase=None, angle=None, phase_dot=None, angle_dot=None):
        """Asynchronous upload of filament state from (preferably pinned) float64 host arrays."""
        def q(a):
            return None if a is None else ctypes.c_void_p(a.ctypes.data if hasattr(a, "ctypes") else a.data_ptr())
        _lib.call("cf_sim_set_state", self._h, q(phase), q(angle), q(phase_dot), q(angle_dot))

    def iteration_log(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.int32)
        _lib.call("cf_sim_iteration_log", self._h, ctypes.c_void_p(out.ctypes.data), int(n))
        return out

    def launches_per_step(self, iters: int) -> int:
        return _lib.load().cf_sim_launches_per_step(self._h, int(iters))

    # -- learned preconditioner (CF_PRECOND_LEARNED) -------------------------
    def learned_dims(self):
        """(feature width, correction width) of the per-filament network."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _lib.call("cf_sim_learned_dims", self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def set_network(self, net):
        """Attaches a FilamentMLP (kept alive by this object) as the learned correction."""
        _lib.call("cf_sim_set_network", self._h, net.handle)
        self._net = net

    def set_network_weight(self, alpha: float):
        """Weight of the network correction (0: the block-diagonal preconditioner alone)."""
        _lib.call("cf_sim_set_network_weight", self._h, ctypes.c_double(alpha))

    def collect_pairs(self, nt: int, max_pairs: int):
        """Runs step nt (block-diagonal handle) and returns the training pairs of its first
        `max_pairs` Arnoldi products as torch CUDA tensors (features [rows, in], targets [rows, out])."""
        import torch
        n_in, n_out = self.learned_dims()
        x = torch.empty((max_pairs * self.n_fil, n_in), dtype=torch.float32, device="cuda")
        t = torch.empty((max_pairs * self.n_fil, n_out), dtype=torch.float32, device="cuda")
        rows = ctypes.c_int()
        _lib.call("cf_sim_collect_pairs", self._h, int(nt), int(max_pairs), ctypes.c_void_p(x.data_ptr()),
                  ctypes.c_void_p(t.data_ptr()), ctypes.byref(rows))
        return x[:rows.value], t[:rows.value]

    def features(self, v) -> np.ndarray:
        """Network features [n_fil, in] of a host vector of the system size."""
        v = np.ascontiguousarray(v, np.float64)
        n_in, _ = self.learned_dims()
        out = np.zeros((self.n_fil, n_in), np.float32)
        _lib.call("cf_sim_features", self._h, _p(v), _p(out))
        return out

    def refresh_preconditioner(self):
        """CF_PRECOND_LINE: rebuilds the patch inverses for the current kinematics (asynchronous)."""
        _lib.call("cf_sim_refresh_preconditioner", self._h)

    def precond_info(self) -> dict:
        np_, mx = ctypes.c_int(), ctypes.c_int()
        fl, by = ctypes.c_double(), ctypes.c_double()
        _lib.call("cf_sim_precond_info", self._h, ctypes.byref(np_), ctypes.byref(mx), ctypes.byref(fl),
                  ctypes.byref(by))
        return dict(patches=np_.value, max_n=mx.value, refresh_flops=fl.value, apply_bytes=by.value)

    def autotune(self, k_hint: int = 0) -> dict:
        """Times the iteration kernels' launch shapes on the current state and keeps the fastest."""
        c = np.zeros(len(_TUNING_KEYS), np.int32)
        _lib.call("cf_sim_autotune", self._h, int(k_hint), ctypes.c_void_p(c.ctypes.data))
        return _tuning_dict(c)

    def tuning(self) -> dict:
        c = np.zeros(len(_TUNING_KEYS), np.int32)
        _lib.call("cf_sim_get_tuning", self._h, ctypes.c_void_p(c.ctypes.data))
        return _tuning_dict(c)

    def set_tuning(self, **kw):
        c = _tuning_array(self.tuning(), kw)
        _lib.call("cf_sim_set_tuning", self._h, ctypes.c_void_p(c.ctypes.data))

    def state(self):
        f = self.n_fil
        ph, an, pd, ad = (np.zeros(f) for _ in range(4))
        _lib.call("cf_sim_get_state", self._h, _p(ph), _p(an), _p(pd), _p(ad))
        return dict(phase=ph, angle=an, phase_dot=pd, angle_dot=ad)

    def solution(self) -> np.ndarray:
        """The saddle-point solution of the last step [system size]: constraint forces, then rates; it is the
        next step's GMRES warm start."""
        out = np.zeros(self.size)
        _lib.call("cf_sim_get_solution", self._h, _p(out))
        return out

    def set_solution(self, sol):
        """Replaces the warm start (and the filament rates, from its rate rows); synchronous."""
        sol = np.ascontiguousarray(sol, np.float64)
        if sol.shape != (self.size,):
            raise ValueError(f"solution must have shape ({self.size},)")
        _lib.call("cf_sim_set_solution", self._h, _p(sol))

    def checkpoint(self) -> dict:
        """Everything the next step depends on: filament state and the warm start."""
        ck = self.state()
        ck["solution"] = self.solution()
        return ck

    def restore(self, ck: dict):
        """Puts back a checkpoint(); the following steps repeat the checkpointed trajectory exactly."""
        self.set_solution(ck["solution"])
        self.set_state(phase=ck["phase"], angle=ck["angle"])

    def segments(self):
        """(x_segs [3N], f_segs [6N]) in the reference's host layouts."""
        x = np.zeros(3 * self.n_seg_total, np.float32)
        fs = np.zeros(6 * self.n_seg_total, np.float32)
        _lib.call("cf_sim_get_segments", self._h, _p(x), _p(fs))
        return x, fs

    def directions(self):
        kp = np.zeros(3 * self.n_seg_total)
        ka = np.zeros(3 * self.n_seg_total)
        _lib.call("cf_sim_get_directions", self._h, _p(kp), _p(ka))
        return kp, ka

    def arclengths(self) -> np.ndarray:
        """Arclength parameters s of the current kinematics, [n_fil, nseg]."""
        out = np.zeros(self.n_seg_total)
        _lib.call("cf_sim_get_arclengths", self._h, _p(out))
        return out.reshape(self.n_fil, self.nseg)

    def tips(self) -> np.ndarray:
        x, _ = self.segments()
        return x.reshape(self.n_fil, self.nseg, 3)[:, -1, :].astype(np.float64)

    def generalised_forces(self):
        """K_phase^T lambda and K_angle^T lambda per filament (cilia_sim_main.cu:420-440)."""
        kp, ka = self.directions()
        _, fs = self.segments()
        lam = fs.reshape(-1, 6)[:, :3].astype(np.float64)
        kp = kp.reshape(-1, 3)
        ka = ka.reshape(-1, 3)
        qp = (kp * lam).sum(1).reshape(self.n_fil, self.nseg).sum(1)
        qa = (ka * lam).sum(1).reshape(self.n_fil, self.nseg).sum(1)
        return qp, qa


def write_generalised_forces_run(beat=_lib.CF_BEAT_FULFORD_BLAKE, nseg=20, seg_sep=2.6, steps=300, tol=1e-8):
    """The reference's WRITE_GENERALISED_FORCES run on the device: one filament with a prescribed
    phase speed of 2 pi per period, arclength by bisection (cilia_sim_main.cu:101-140, 318-338, 420-440).
    Returns (phase forces [steps], angle forces [steps])."""
    qp = np.zeros(steps)
    qa = np.zeros(steps)
    with WallCiliaSimulation(bases=[[0.0, 0.0, 0.5 * seg_sep]], nseg=nseg, seg_sep=seg_sep, beat=beat,
                             dt=1.0 / steps, dynamic_phase=False, dynamic_angle=False, gmres_tol=tol) as sim:
        for nt in range(steps):
            sim.step(nt)
            a, b = sim.generalised_forces()
            qp[nt], qa[nt] = a[0], b[0]
    return qp, qa


def arclength_table(beat=_lib.CF_BEAT_FULFORD_BLAKE, nseg=20, seg_sep=2.6, steps=300, tol_factor=0.0):
    """Arclength parameters over one period [steps, nseg], as the reference's WRITE_GENERALISED_FORCES
    run writes its s_values file (phase advancing by 2 pi/steps per step, bisection on the device)."""
    out = np.zeros((steps, nseg))
    with WallCiliaSimulation(bases=[[0.0, 0.0, 0.5 * seg_sep]], nseg=nseg, seg_sep=seg_sep, beat=beat,
                             dt=1.0 / steps, dynamic_phase=False, dynamic_angle=False, gmres_tol=1e-3,
                             s_tol_factor=tol_factor) as sim:
        for nt in range(steps):
            sim.initial_guess(nt)
            out[nt] = sim.arclengths()[0]
    return out


_TUNING_KEYS = ("pair_ctas_per_sm", "dots_chunk", "dots_blocks_per_sm", "update_blocks_per_sm", "update_rows")


def _tuning_dict(c) -> dict:
    return {k: int(v) for k, v in zip(_TUNING_KEYS, c)}


def _tuning_array(cur: dict, kw: dict) -> np.ndarray:
    unknown = set(kw) - set(_TUNING_KEYS)
    if unknown:
        raise ValueError(f"unknown tuning keys {sorted(unknown)}")
    cur = dict(cur, **kw)
    return np.asarray([cur[k] for k in _TUNING_KEYS], np.int32)


class WallCiliaBatch:
    """Many independent wall arrays of uneven size stepped together (cf_batch).

    ``arrays`` is a list of per-array keyword dicts for the array-specific
    settings (``bases`` and optionally ``omega0``, ``phase0``, ``angle0``);
    every other setting is shared and given as keyword arguments, with the
    same meaning as for :class:`WallCiliaSimulation`.  Each array runs its own
    GMRES; per-array results come back as arrays of length ``n_arrays`` and
    per-filament state is split into one array per cilia array."""

    def __init__(self, arrays, nseg=20, **shared):
        self._keep = []
        cfgs = (_lib.SimConfig * len(arrays))()
        self.n_fils = []
        for b, spec in enumerate(arrays):
            merged = dict(shared, **spec)
            merged.setdefault("nseg", nseg)
            cfgs[b] = _sim_config(self._keep, **merged)
            self.n_fils.append(cfgs[b].n_fil)
        self.n_arrays = len(arrays)
        self.nseg = int(nseg)
        h = ctypes.c_void_p()
        _lib.call("cf_batch_create", cfgs, len(arrays), ctypes.byref(h))
        self._h = h
        sizes = np.zeros(self.n_arrays, np.int32)
        nf, ns = ctypes.c_int(), ctypes.c_int()
        _lib.call("cf_batch_shape", self._h, None, ctypes.byref(nf), ctypes.byref(ns), _p(sizes))
        self.sizes = sizes
        self.n_fil_total = nf.value
        self.n_seg_total = ns.value
        self._fil_split = np.cumsum(self.n_fils)[:-1]

    def close(self):
        if getattr(self, "_h", None):
            _lib.call("cf_batch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, nt: int):
        """One implicit step of every array; returns (iterations, relative residuals, status code)."""
        it = np.zeros(self.n_arrays, np.int32)
        rel = np.zeros(self.n_arrays)
        rc = _lib.call("cf_batch_step", self._h, int(nt), _p(it), _p(rel),
                       ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED))
        return it, rel, rc

    def step_async(self, nt: int):
        _lib.call("cf_batch_step_async", self._h, int(nt))

    def last_solve(self):
        """(iterations, relative residuals, per-array GMRES status, worst status code)."""
        it = np.zeros(self.n_arrays, np.int32)
        rel = np.zeros(self.n_arrays)
        st = np.zeros(self.n_arrays, np.int32)
        rc = _lib.call("cf_batch_last_solve", self._h, _p(it), _p(rel), _p(st),
                       ok=(_lib.CF_OK, _lib.CF_NOT_CONVERGED, _lib.CF_NONFINITE))
        return it, rel, st, rc

    def state(self):
        """Filament state, one list entry per array: dicts of phase, angle, phase_dot, angle_dot."""
        f = self.n_fil_total
        ph, an, pd, ad = (np.zeros(f) for _ in range(4))
        _lib.call("cf_batch_get_state", self._h, _p(ph), _p(an), _p(pd), _p(ad))
        parts = [np.split(a, self._fil_split) for a in (ph, an, pd, ad)]
        return [dict(phase=p, angle=a, phase_dot=q, angle_dot=r) for p, a, q, r in zip(*parts)]

    def set_state(self, phase=None, angle=None, phase_dot=None, angle_dot=None):
        """Per-filament state concatenated over the arrays (float64; any may be None)."""
        keep = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (phase, angle, phase_dot,
                                                                                      angle_dot)]
        _lib.call("cf_batch_set_state", self._h, *(_p(a) for a in keep))
        _lib.call("cf_batch_get_state", self._h, None, None, None, None)  # waits for the uploads

    def segments(self):
        """Segment positions per array, [n_fil * nseg, 3] float64 each."""
        x = np.zeros(3 * self.n_seg_total)
        _lib.call("cf_batch_get_segments", self._h, _p(x))
        x = x.reshape(-1, 3)
        return np.split(x, np.cumsum(self.n_fils)[:-1] * self.nseg)

    def tips(self):
        return [s.reshape(-1, self.nseg, 3)[:, -1, :] for s in self.segments()]

    def solution(self, array: int) -> np.ndarray:
        out = np.zeros(int(self.sizes[array]))
        _lib.call("cf_batch_get_solution", self._h, int(array), _p(out))
        return out

    def iteration_log(self, array: int, n: int) -> np.ndarray:
        out = np.zeros(n, np.int32)
        _lib.call("cf_batch_iteration_log", self._h, int(array), _p(out), int(n))
        return out

    def stream_handle(self) -> int:
        h = ctypes.c_void_p()
        _lib.call("cf_batch_stream", self._h, ctypes.byref(h))
        return h.value or 0

    def launches_per_step(self, loop_iters: int) -> int:
        return _lib.load().cf_batch_launches_per_step(self._h, int(loop_iters))

    def autotune(self, k_hint: int = 0) -> dict:
        c = np.zeros(len(_TUNING_KEYS), np.int32)
        _lib.call("cf_batch_autotune", self._h, int(k_hint), _p(c))
        return _tuning_dict(c)

    def tuning(self) -> dict:
        c = np.zeros(len(_TUNING_KEYS), np.int32)
        _lib.call("cf_batch_get_tuning", self._h, _p(c))
        return _tuning_dict(c)

    def set_tuning(self, **kw):
        c = _tuning_array(self.tuning(), kw)
        _lib.call("cf_batch_set_tuning", self._h, _p(c))


def lattice_simulation(nx: int = 16, *, spacing: float = 20.0, nseg: int = 20, seg_sep: float = 2.6, seed: int = 2024,
                       s_table=None, **kw) -> WallCiliaSimulation:
    """The benchmark array: nx x nx Fulford-Blake cilia on a square wall lattice (bases at z = seg_sep/2),
    phases U(0, 2 pi) and angles N(0, 0.05) from `seed`, dt = T/300, spring factor 0.01, the reference's
    generalised-force tables and the device-generated arclength table; other keywords go to
    WallCiliaSimulation (precond, gmres_tol, line_patch, device, ...)."""
    from pathlib import Path
    from . import workloads
    data = np.load(Path(__file__).resolve().parent / "data" / "fulford_blake_nseg20_sep2.6.npz")
    F = nx * nx
    rng = np.random.default_rng(seed)
    phase0 = rng.uniform(0.0, 2.0 * math.pi, F)
    angle0 = rng.normal(0.0, 0.05, F)
    if s_table is None:
        s_table = arclength_table(nseg=nseg, seg_sep=seg_sep, steps=300)
    args = dict(nseg=nseg, seg_sep=seg_sep, dt=1.0 / 300, phase0=phase0, angle0=angle0, spring_factor=0.01,
                phase_refs=data["phase"], angle_refs=data["angle"], s_table=s_table)
    args.update(kw)
    return WallCiliaSimulation(bases=workloads.lattice_bases(F, nx, spacing, 0.5 * seg_sep), **args)

