"""Python owner of one native solver handle (libsoliton_b200).

``Solver`` creates the handle from the reference's packed ``p_i``/``p_f`` arrays,
allocates the caller-owned device workspace as a torch tensor and forwards every
call to the C ABI on the bound CUDA stream.  Device buffers are torch tensors (or
anything exposing ``data_ptr()``); they must be contiguous, on the solver's
device and of the solver's element type.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from soliton_solver_b200 import _native as nat

_CHARGES = {"skyrmion": nat.SS_CHARGE_SKYRMION, "magnetic": nat.SS_CHARGE_MAGNETIC, "vortex": nat.SS_CHARGE_VORTEX}
_DENSITIES = {"higgs": nat.SS_DENSITY_HIGGS, "higgs1": nat.SS_DENSITY_HIGGS1, "higgs2": nat.SS_DENSITY_HIGGS2,
              "phase": nat.SS_DENSITY_PHASE_DIFFERENCE, "supercurrent": nat.SS_DENSITY_SUPERCURRENT,
              "magnetic": nat.SS_DENSITY_MAGNETIC_FIELD}
_COUPLINGS = {"kappa": nat.SS_COUPLING_KAPPA, "mpi": nat.SS_COUPLING_MPI, "Lambda": nat.SS_COUPLING_LAMBDA,
              "coup_K": nat.SS_COUPLING_COUP_K, "coup_h": nat.SS_COUPLING_COUP_H,
              "coup_mu": nat.SS_COUPLING_COUP_MU}


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, torch.Tensor):
        return t.data_ptr()
    cai = getattr(t, "__cuda_array_interface__", None)
    if cai is not None:
        return int(cai["data"][0])
    raise TypeError(f"expected a CUDA tensor, got {type(t)!r}")


class Solver:
    """One lattice of one theory on one CUDA device."""

    def __init__(self, theory_id: int, p_i, p_f, precision: str = "fp32", device=None, stream=None):
        lib = nat.load()
        if precision not in nat.PRECISIONS:
            raise ValueError(f"precision must be one of {tuple(nat.PRECISIONS)}")
        self.precision = precision
        self.dtype = torch.float32 if precision == "fp32" else torch.float64
        self.p_i = np.ascontiguousarray(p_i, dtype=np.int32)
        self.p_f = np.ascontiguousarray(p_f, dtype=np.float64)
        self.theory_id = int(theory_id)
        self.xlen, self.ylen, self.nf = int(self.p_i[0]), int(self.p_i[1]), int(self.p_i[4])
        self.N = self.xlen * self.ylen
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        nat.check(lib.ss_create(self.theory_id, self.p_i.ctypes.data, len(self.p_i), self.p_f.ctypes.data,
                                len(self.p_f), nat.PRECISIONS[precision], ctypes.byref(h)))
        self._h = h
        self._lib = lib
        nbytes = ctypes.c_size_t()
        nat.check(lib.ss_workspace_bytes(h, ctypes.byref(nbytes)))
        self.workspace = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        self.field = None
        self.velocity = None
        self.stream = stream
        self._bind(None, None)

    # ------------------------------------------------------------------ binding
    def _stream_handle(self):
        if self.stream is not None:
            return int(self.stream.cuda_stream) if hasattr(self.stream, "cuda_stream") else int(self.stream)
        return int(torch.cuda.current_stream(self.device).cuda_stream)

    def _bind(self, field, velocity):
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_bind(self._h, _ptr(field), _ptr(velocity), self.workspace.data_ptr(),
                                        self.workspace.numel(), self._stream_handle()))
        self.field, self.velocity = field, velocity

    def bind(self, field: torch.Tensor, velocity: torch.Tensor):
        """Bind the Field/Velocity buffers that ``step`` advances in place."""
        self._check(field)
        self._check(velocity)
        self._bind(field, velocity)

    def _check(self, t, dtype=None):
        if not isinstance(t, torch.Tensor):
            return
        want = dtype or self.dtype
        if t.dtype != want or t.device != self.device or not t.is_contiguous():
            raise ValueError(f"buffer must be a contiguous {want} tensor on {self.device}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and getattr(self, "_lib", None) is not None:
            try:
                self._lib.ss_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------------ flow
    def step(self, n_steps: int = 1, prev_energy: float = math.nan):
        """Advance the bound buffers; returns (energy_traj, err_traj) numpy arrays."""
        E = np.empty(max(n_steps, 0))
        err = np.empty(max(n_steps, 0))
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_step(self._h, int(n_steps), float(prev_energy), E.ctypes.data, err.ctypes.data))
        return E, err

    def step_async(self, n_steps: int, prev_energy: float = math.nan, energy_traj=None, err_traj=None):
        """Advance without a host synchronisation; trajectories go to device tensors."""
        for t in (energy_traj, err_traj):
            if t is not None:
                self._check(t, torch.float64)
                if t.numel() < n_steps:
                    raise ValueError("trajectory buffer shorter than n_steps")
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_step_async(self._h, int(n_steps), float(prev_energy), _ptr(energy_traj),
                                              _ptr(err_traj)))

    def capture(self, n_steps: int, energy_traj=None, err_traj=None):
        """Capture n_steps of step_async into a CUDA graph (replay with replay())."""
        for t in (energy_traj, err_traj):
            if t is not None:
                self._check(t, torch.float64)
                if t.numel() < n_steps:
                    raise ValueError("trajectory buffer shorter than n_steps")
        self._graph_bufs = (energy_traj, err_traj)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_graph_create(self._h, int(n_steps), _ptr(energy_traj), _ptr(err_traj)))

    def replay(self):
        """Launch the captured graph on the bound stream (no host synchronisation)."""
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_graph_launch(self._h))

    @property
    def tma_enabled(self) -> bool:
        """True when the bound buffers are staged with TMA tensor maps."""
        return bool(self._lib.ss_tma_enabled(self._h))

    def autotune(self, iters: int = 5):
        """Pick the faster TMA staging variant of each flow stage on the bound buffers.

        Returns {stage: (ms one-tile-per-CTA, ms pipelined, chosen)} for stages 1-4 and
        {6: (ms stages 2 and 3 as two kernels, ms fused, 1 if fused)}."""
        ms = np.zeros(14, dtype=np.float32)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_autotune(self._h, int(iters), ms.ctypes.data))
        return {m: (float(ms[2 * m]), float(ms[2 * m + 1]), int(self._lib.ss_get_variant(self._h, m)))
                for m in (1, 2, 3, 4, 6)}

    def initialize(self, field, velocity=None, mode: int = nat.SS_INIT_GROUND, ansatz: int = nat.SS_ANSATZ_BLOCH,
                   rotation: float = 0.0, vortex_number: float = 1.0):
        """Ground state or single-soliton ansatz into `field` (velocity zeroed if given);
        see ss_initialize.  Asynchronous on the solver's stream."""
        self._check(field)
        if velocity is not None:
            self._check(velocity)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_initialize(self._h, _ptr(field), _ptr(velocity), int(mode), int(ansatz),
                                              float(rotation), float(vortex_number)))

    def insert_soliton(self, field, pxi: int, pxj: int, ansatz: int = nat.SS_ANSATZ_BLOCH, vortex: int = 1,
                       rotation: float = 0.0):
        """Add a skyrmion (chiral magnet, baby Skyrme) or a vortex (Abelian Higgs, s+id)
        centred on lattice point (pxi, pxj) to `field`; see ss_insert_soliton."""
        self._check(field)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_insert_soliton(self._h, _ptr(field), int(pxi), int(pxj), int(ansatz),
                                                  int(vortex), float(rotation)))

    def set_variant(self, stage: int, variant: int):
        """Pin the staging variant of flow mode `stage` (0 gradient, 1-4 stages):
        0 one tile per CTA, 1 pipelined (see ss_set_variant)."""
        nat.check(self._lib.ss_set_variant(self._h, int(stage), int(variant)))

    def debug_wait_timeout(self, wait_cycles: int, inject: bool):
        """Failure-detection hook: bound of the device waits; optionally make the next
        stage kernel's wait expire (see ss_debug_wait_timeout)."""
        nat.check(self._lib.ss_debug_wait_timeout(self._h, int(wait_cycles), 1 if inject else 0))

    def rebind(self):
        """Re-bind the current buffers (resets the device step state)."""
        self._bind(self.field, self.velocity)

    def check_status(self):
        nat.check(self._lib.ss_check_status(self._h))

    # ------------------------------------------------------------------ hooks
    def gradient(self, field, energy_gradient=None, l_out=None):
        for t in (field, energy_gradient, l_out):
            if t is not None:
                self._check(t)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_gradient(self._h, _ptr(field), _ptr(energy_gradient), _ptr(l_out)))

    def energy_gradient(self, field, out=None):
        """dE/dphi per site (unprojected; see ss_energy_gradient)."""
        self._check(field)
        out = out if out is not None else torch.empty_like(field)
        self._check(out)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_energy_gradient(self._h, _ptr(field), _ptr(out)))
        return out

    def energy_gradient_exact(self, field, out=None, minus_stencil: bool = False):
        """dE_h/dphi / dA of the discrete energy sum, exactly (true rows, unprojected;
        see ss_energy_gradient_exact), FP64; with `minus_stencil` (FP64 solvers) minus the
        flow's functional derivative: the O(h^4) discretisation residual.  Uses the
        workspace's flow buffers: not during a step."""
        self._check(field)
        out = out if out is not None else torch.empty(self.nf * self.N, dtype=torch.float64, device=self.device)
        self._check(out, torch.float64)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_energy_gradient_exact(self._h, _ptr(field), _ptr(out), 1 if minus_stencil else 0))
        return out

    def set_forcing(self, force=None):
        """Add the fixed FP64 field `force` (true rows) to the flow's gradient in every
        following step (None removes it); see ss_set_forcing.  The tensor is kept alive
        while it is set."""
        if force is not None:
            self._check(force, torch.float64)
            if force.numel() != self.nf * self.N:
                raise ValueError("forcing must have nf * N entries")
        nat.check(self._lib.ss_set_forcing(self._h, _ptr(force)))
        self._force = force

    def energy(self, field) -> float:
        self._check(field)
        out = ctypes.c_double()
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_energy(self._h, _ptr(field), ctypes.byref(out)))
        return out.value

    def energy_projected(self, field) -> float:
        """FP64 energy of `field` with each site's unit vector renormalised in FP64
        (ss_energy_projected).  Uses the workspace's l buffers: not during a step."""
        self._check(field)
        out = ctypes.c_double()
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_energy_projected(self._h, _ptr(field), ctypes.byref(out)))
        return out.value

    def energy_density(self, field, out=None):
        self._check(field)
        out = out if out is not None else torch.empty(self.N, dtype=torch.float64, device=self.device)
        self._check(out, torch.float64)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_energy_density(self._h, _ptr(field), _ptr(out)))
        return out

    def charge(self, field, which: str) -> float:
        self._check(field)
        out = ctypes.c_double()
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_charge(self._h, _ptr(field), _CHARGES[which], ctypes.byref(out)))
        return out.value

    def charge_density(self, field, which: str, out=None):
        self._check(field)
        out = out if out is not None else torch.empty(self.N, dtype=torch.float64, device=self.device)
        self._check(out, torch.float64)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_charge_density(self._h, _ptr(field), _CHARGES[which], _ptr(out)))
        return out

    def convert(self, src, dst, project: bool = True):
        """Copy `src` into `dst` (FP32 or FP64 tensors of this lattice, either way round),
        with each site's unit vector renormalised in FP64 first when `project` (see
        ss_convert_field).  Asynchronous on the solver's stream."""
        for t in (src, dst):
            if not isinstance(t, torch.Tensor) or t.dtype not in (torch.float32, torch.float64) or \
                    t.device != self.device or not t.is_contiguous() or t.numel() != self.nf * self.N:
                raise ValueError(f"convert needs contiguous FP32/FP64 tensors of {self.nf * self.N} entries on "
                                 f"{self.device}")
        code = {torch.float32: nat.SS_FP32, torch.float64: nat.SS_FP64}
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_convert_field(self._h, _ptr(src), code[src.dtype], _ptr(dst), code[dst.dtype],
                                                 1 if project else 0))
        return dst

    def field_density(self, field, kind: str, out=None):
        """Diagnostic density of a gauge theory (see ss_field_density): 'higgs', 'higgs1',
        'higgs2', 'phase', 'magnetic' (N doubles) or 'supercurrent' (2 N: x plane, y plane).
        Asynchronous on the solver's stream."""
        self._check(field)
        n = 2 * self.N if kind == "supercurrent" else self.N
        out = out if out is not None else torch.empty(n, dtype=torch.float64, device=self.device)
        self._check(out, torch.float64)
        if out.numel() < n:
            raise ValueError(f"output buffer needs {n} entries")
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_field_density(self._h, _ptr(field), _DENSITIES[kind], _ptr(out)))
        return out

    def coupling_grad(self, field, which: str) -> float:
        self._check(field)
        out = ctypes.c_double()
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_coupling_grad(self._h, _ptr(field), _COUPLINGS[which], ctypes.byref(out)))
        return out.value

    def rk4_stage(self, k_out, velocity, l_in, temp, field, k_prev, factor: float):
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_rk4_stage(self._h, _ptr(k_out), _ptr(velocity), _ptr(l_in), _ptr(temp),
                                             _ptr(field), _ptr(k_prev), float(factor)))

    def rk4_finalize(self, velocity, field, k1, k2, k3, k4, l1, l2, l3, l4):
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_rk4_finalize(self._h, _ptr(velocity), _ptr(field), *(
                _ptr(t) for t in (k1, k2, k3, k4, l1, l2, l3, l4))))


_CACHE: dict = {}


def solver_for(theory_id: int, p_i, p_f, dtype, device) -> Solver:
    """Cached solver for hook-style calls that pass packed parameter arrays."""
    p_i = np.ascontiguousarray(_to_host(p_i), dtype=np.int32)
    p_f = np.ascontiguousarray(_to_host(p_f), dtype=np.float64)
    precision = "fp32" if dtype == torch.float32 else "fp64"
    key = (theory_id, precision, str(device), p_i.tobytes(), p_f.tobytes())
    s = _CACHE.get(key)
    if s is None:
        if len(_CACHE) > 64:
            _CACHE.clear()
        s = Solver(theory_id, p_i, p_f, precision, device)
        _CACHE[key] = s
    return s


def _to_host(a):
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    if hasattr(a, "copy_to_host"):
        return a.copy_to_host()
    return np.asarray(a)
