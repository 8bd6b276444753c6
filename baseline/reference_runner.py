"""Run the unmodified reference soliton_solver (installed into baseline/_ref) on the host.

The reference's numerics are Numba CUDA kernels.  On the host they run under Numba's
CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``), which executes every kernel thread as
Python code: the reference's own CPU path.  Each worker process imports the
reference from ``baseline/_ref`` through its public API (``load_theory``,
``theory.params.default_params``, ``Simulation``, ``sim.initialize``,
``sim.step``) with empty stand-in modules for the viewer's window/GL imports
(``glfw``, ``OpenGL*``, ``moderngl``), so that the theory packages register; no
viewer code runs.  Nothing of this repository's library is imported by a worker.

The install is one offline command (from a copy of the reference checkout, since
the build writes into the source tree):

    python -m pip install --no-index --no-build-isolation --no-deps \
        --find-links /opt/wheelhouse --target baseline/_ref <copy of the reference>

``--no-deps``: the reference's viewer dependencies (moderngl, glfw, PyOpenGL) and
numba-cuda have no wheels offline; numba's built-in CUDA target (numba 0.65) serves.

``time_flow_steps`` measures whole ``Simulation.step(prev_energy)`` calls on a
sub-lattice of the chiral-magnet workload in ``n_proc`` independent processes (the
simulator holds the GIL, so one process uses one core).  ``numba_gpu_flow_steps`` runs
the same reference code on Numba's real CUDA target (for the GPU comparator).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
STUBS = ("glfw", "OpenGL", "OpenGL.GL", "OpenGL.GL.shaders", "OpenGL.GLUT", "moderngl")


def available() -> str | None:
    """None when the reference is installed, else the reason it is not."""
    if not os.path.isdir(os.path.join(REF_DIR, "soliton_solver")):
        return "reference not installed into baseline/_ref (see baseline/reference_runner.py)"
    try:
        import numba  # noqa: F401
    except Exception as exc:  # pragma: no cover - numba is part of the image
        return f"numba unavailable: {exc}"
    return None


def _import_reference(simulator: bool):
    if simulator:
        os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    else:
        os.environ.pop("NUMBA_ENABLE_CUDASIM", None)
    for name in STUBS:
        sys.modules.setdefault(name, types.ModuleType(name))
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import numpy as np
    from numba import cuda
    from soliton_solver.core.simulation import Simulation
    from soliton_solver.theories import load_theory
    return np, cuda, load_theory, Simulation


def _workload_params(load_theory, n, spacing, B, demag):
    """The chiral-magnet workload's couplings on an n x n lattice with the workload's spacing."""
    th = load_theory("Chiral magnet")
    size = spacing * (n - 1)
    p = th.params.default_params(xlen=n, ylen=n, xsize=size, ysize=size, J=40e-12, K=0.8e6, D=4e-3, M=580e3,
                                 B=B, dmi_term="Heusler", demag=demag, unit_magnetization=True, killkinen=True)
    return th, p


def _ground_plus_noise(np, sim, seed):
    """The reference's ground state plus N(0, 1e-3) noise, renormalised (numpy, host side)."""
    F = sim.Field.copy_to_host().reshape(sim.rp.number_total_fields, sim.rp.xlen, sim.rp.ylen)
    F = F + 1e-3 * np.random.default_rng(seed).standard_normal(F.shape)
    F[:3] /= np.sqrt((F[:3] ** 2).sum(0))
    sim.Field.copy_to_device(np.ascontiguousarray(F.reshape(-1)))


def _worker(job):
    n, spacing, B, demag, steps, warmup, seed = job
    np, cuda, load_theory, Simulation = _import_reference(simulator=True)
    th, p = _workload_params(load_theory, n, spacing, B, demag)
    sim = Simulation(p, th)
    sim.initialize({"mode": "ground"})
    _ground_plus_noise(np, sim, seed)
    E = 1e300
    for _ in range(warmup):
        E, _ = sim.step(E)
    t = time.perf_counter()
    for _ in range(steps):
        E, _ = sim.step(E)
    return (time.perf_counter() - t) / max(steps, 1), float(E)


def time_flow_steps(n=16, spacing=128.0 / 4095, B=0.2, demag=True, steps=2, warmup=1, n_proc=None):
    """Seconds per reference ``Simulation.step`` on an n x n sub-lattice of the workload,
    in ``n_proc`` independent processes at once (spawned; each one core).  Returns
    (point-updates/s over all processes, n_proc, mean s/step, energies)."""
    n_proc = n_proc or max(1, min(os.cpu_count() or 1, 32))
    jobs = [(n, spacing, B, demag, steps, warmup, seed) for seed in range(n_proc)]
    with mp.get_context("spawn").Pool(n_proc) as pool:
        res = pool.map(_worker, jobs)
    per_step = [r[0] for r in res]
    value = sum(n * n / s for s in per_step)
    return value, n_proc, sum(per_step) / len(per_step), [r[1] for r in res]


def numba_gpu_flow_steps(n=512, steps=20, warmup=2):
    """The reference's own Simulation.step on Numba's real CUDA target (FP64 kernels,
    host-side arrest), n x n sub-lattice of the workload.  Run in a process of its own.
    Returns a dict with seconds per step or the error the target raised."""
    try:
        np, cuda, load_theory, Simulation = _import_reference(simulator=False)
        th, p = _workload_params(load_theory, n, 128.0 / 4095, 0.2, True)
        sim = Simulation(p, th)
        sim.initialize({"mode": "ground"})
        _ground_plus_noise(np, sim, 0)
        E = 1e300
        for _ in range(warmup):
            E, _ = sim.step(E)
        cuda.synchronize()
        t = time.perf_counter()
        for _ in range(steps):
            E, _ = sim.step(E)
        cuda.synchronize()
        dt = (time.perf_counter() - t) / steps
        return {"ok": True, "n": n, "steps": steps, "s_per_step": dt, "point_updates_per_s": n * n / dt,
                "energy": float(E), "device": cuda.get_current_device().name.decode()
                if isinstance(cuda.get_current_device().name, bytes) else str(cuda.get_current_device().name)}
    except Exception as exc:  # the target may not support this GPU: report, do not fail
        return {"ok": False, "error": f"{type(exc).__name__}: {str(exc).splitlines()[0] if str(exc) else ''}"}


if __name__ == "__main__":
    import json
    if len(sys.argv) > 1 and sys.argv[1] == "gpu":
        print(json.dumps(numba_gpu_flow_steps(int(sys.argv[2]) if len(sys.argv) > 2 else 512,
                                              int(sys.argv[3]) if len(sys.argv) > 3 else 20)))
    else:
        print(json.dumps(time_flow_steps(n_proc=int(sys.argv[1]) if len(sys.argv) > 1 else 2)))
