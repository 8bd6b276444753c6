"""Many independent relaxations of one theory, advanced together.

``BatchSolver`` owns one native batch (ss_batch_*): every lattice has its own size,
couplings, Field/Velocity buffers, energy and arrest state, and one launch per RK
stage covers all of them.  Each lattice's step is exactly what a single-lattice
``Solver`` would do.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from soliton_solver_b200 import _native as nat


class BatchSolver:
    def __init__(self, theory, params_list, precision: str = "fp32", device=None):
        if precision not in ("fp32", "fp64"):
            raise ValueError("batches support fp32 and fp64")
        lib = nat.load()
        self._lib = lib
        self.theory = theory
        self.precision = precision
        self.dtype = torch.float32 if precision == "fp32" else torch.float64
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.rps = [p.resolved() if hasattr(p, "resolved") else p for p in params_list]
        packs = [theory.params.pack_device_params(rp) for rp in self.rps]
        self.p_i = np.ascontiguousarray(np.stack([p[0] for p in packs]), dtype=np.int32)
        self.p_f = np.ascontiguousarray(np.stack([p[1] for p in packs]), dtype=np.float64)
        self.n = len(self.rps)
        h = ctypes.c_void_p()
        nat.check(lib.ss_batch_create(theory.kernels.THEORY_ID, self.n, self.p_i.ctypes.data, self.p_i.shape[1],
                                      self.p_f.ctypes.data, self.p_f.shape[1], nat.PRECISIONS[precision],
                                      ctypes.byref(h)))
        self._h = h
        nbytes = ctypes.c_size_t()
        nat.check(lib.ss_batch_workspace_bytes(h, ctypes.byref(nbytes)))
        self.workspace = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        self.fields = [torch.zeros(int(rp.dim_fields), dtype=self.dtype, device=self.device) for rp in self.rps]
        self.velocities = [torch.zeros_like(f) for f in self.fields]
        fp = (ctypes.c_void_p * self.n)(*[f.data_ptr() for f in self.fields])
        vp = (ctypes.c_void_p * self.n)(*[v.data_ptr() for v in self.velocities])
        stream = int(torch.cuda.current_stream(self.device).cuda_stream)
        with torch.cuda.device(self.device):
            nat.check(lib.ss_batch_bind(h, fp, vp, self.workspace.data_ptr(), self.workspace.numel(), stream))

    @property
    def tma_enabled(self) -> bool:
        return bool(self._lib.ss_batch_tma_enabled(self._h))

    def autotune(self, iters: int = 3):
        """Pick the tile shape of every size class (lattices of equal extents) by timing
        one step's stage launches in each shape (see ss_batch_autotune).  Returns
        {(xlen, ylen): (ms in 16 x 64 tiles, ms in 8 x 32 tiles, chosen shape)}."""
        ms = np.zeros(2 * self.n, dtype=np.float32)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_batch_autotune(self._h, int(iters), ms.ctypes.data))
        out = {}
        for i, rp in enumerate(self.rps):
            out[(int(rp.xlen), int(rp.ylen))] = (float(ms[2 * i]), float(ms[2 * i + 1]), self.shape(i))
        return out

    def shape(self, i: int) -> int:
        """Tile shape of lattice i: 0 (16 x 64 sites) or 1 (8 x 32)."""
        return int(self._lib.ss_batch_get_shape(self._h, int(i)))

    def set_shape(self, i: int, shape: int):
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_batch_set_shape(self._h, int(i), int(shape)))

    def load(self, i: int, field, velocity=None):
        f = torch.as_tensor(np.asarray(field) if not isinstance(field, torch.Tensor) else field)
        self.fields[i].copy_(f.reshape(-1).to(self.dtype))
        if velocity is None:
            self.velocities[i].zero_()
        else:
            v = torch.as_tensor(np.asarray(velocity) if not isinstance(velocity, torch.Tensor) else velocity)
            self.velocities[i].copy_(v.reshape(-1).to(self.dtype))

    def step(self, n_steps: int, prev_energy=None):
        """Advance every lattice; returns (energy_traj, err_traj) of shape (n_lattices, n_steps)."""
        E = np.empty((self.n, max(n_steps, 0)))
        err = np.empty((self.n, max(n_steps, 0)))
        prev = None
        if prev_energy is not None:
            prev = np.ascontiguousarray(np.broadcast_to(np.asarray(prev_energy, dtype=np.float64), (self.n,)))
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_batch_step(self._h, int(n_steps), None if prev is None else prev.ctypes.data,
                                              E.ctypes.data, err.ctypes.data))
        return E, err

    def capture(self, n_steps: int):
        """Capture n_steps (<= 1024) of every lattice into a CUDA graph."""
        self._graph_steps = int(n_steps)
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_batch_graph_create(self._h, int(n_steps)))

    def replay(self):
        with torch.cuda.device(self.device):
            nat.check(self._lib.ss_batch_graph_launch(self._h))

    def trajectory(self):
        """(energy, err) of the last graph replay, shape (n_lattices, captured steps)."""
        n = self._graph_steps
        E = np.empty((self.n, n))
        err = np.empty((self.n, n))
        nat.check(self._lib.ss_batch_trajectory(self._h, n, E.ctypes.data, err.ctypes.data))
        return E, err

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None:
            try:
                self._lib.ss_batch_destroy(h)
            except Exception:
                pass
            self._h = None
