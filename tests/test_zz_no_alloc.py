"""The allocation-free energy entry point, ss_energy_noalloc.

It serves callers that cannot allocate device memory when they need an energy: a
host whose memory manager owns all device memory, or an interactive loop that must
not call cudaMalloc/cudaFree because they synchronise the device.  Its scratch is a
static device array.  Here it is called through the C ABI twice in a row, on two
different fields, and each result is compared with the existing ss_energy entry
point (which uses a caller-allocated workspace) at the tolerance the other energy
tests use (1e-10 relative); the device's free memory and torch's allocations are
unchanged across the calls; a lattice of exactly the maximum tile count, whose last
partial sits at the end of the array, matches too.  This file is collected last on
purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from soliton_solver_b200 import _native as nat
from soliton_solver_b200.core.solver import Solver
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu


def _field(rp, seed, dtype):
    rng = np.random.default_rng(seed)
    X, Y, nf = rp.xlen, rp.ylen, rp.number_total_fields
    F = 0.2 * rng.standard_normal((nf, X, Y))
    F[2] += 1.0
    if nf >= 3 and getattr(rp, "unit_magnetization", 0):
        F[:3] /= np.sqrt((F[:3] ** 2).sum(0))
    return torch.tensor(F.reshape(-1), dtype=dtype, device="cuda")


def _noalloc_energy(theory_id, p_i, p_f, precision, field):
    lib = nat.load()
    out = ctypes.c_double(np.nan)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.ss_energy_noalloc(theory_id, p_i.ctypes.data, len(p_i), p_f.ctypes.data, len(p_f),
                               nat.PRECISIONS[precision], field.data_ptr(), ctypes.byref(out), stream)
    nat.check(rc)
    return out.value


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("name,kw", [
    ("Chiral magnet", dict(xlen=300, ylen=260, xsize=9.0, ysize=7.8, dmi_term="Heusler", demag=True, B=0.2,
                           unit_magnetization=True)),
    ("Abelian Higgs", dict(xlen=129, ylen=131, xsize=6.4, ysize=6.5, Lambda=0.7)),
])
def test_noalloc_energy_matches_workspace_energy_twice(name, kw, precision):
    theory = load_theory(name)
    rp = theory.params.default_params(**kw).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    dtype = torch.float32 if precision == "fp32" else torch.float64
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, precision)
    fields = [_field(rp, seed, dtype) for seed in (1, 2)]
    want = [s.energy(f) for f in fields]
    _noalloc_energy(theory.kernels.THEORY_ID, p_i, p_f, precision, fields[0])  # loads the module
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    # two calls in a row: the static scratch keeps the previous call's contents
    got = [_noalloc_energy(theory.kernels.THEORY_ID, p_i, p_f, precision, f) for f in fields]
    assert torch.cuda.mem_get_info()[0] == free0 and torch.cuda.memory_allocated() == alloc0
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-10 * max(1.0, abs(w)), (g, w)


def test_noalloc_energy_at_the_maximum_tile_count():
    """512 x 131008 sites = 32 x 2047 = 65504 tiles of 16 x 64, the largest lattice the
    static scratch takes: its last partial fills the array's last slot."""
    theory = load_theory("Baby Skyrme")
    rp = theory.params.default_params(xlen=512, ylen=131008, lsx=0.1, lsy=0.1, unit_magnetization=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    g = torch.Generator(device="cuda").manual_seed(7)
    f = 0.2 * torch.randn(3, rp.xlen * rp.ylen, device="cuda", generator=g)
    f[2] += 1.0
    f = (f / f.norm(dim=0)).reshape(-1).contiguous()
    want = Solver(theory.kernels.THEORY_ID, p_i, p_f, "fp32").energy(f)
    for _ in range(2):
        got = _noalloc_energy(theory.kernels.THEORY_ID, p_i, p_f, "fp32", f)
        assert abs(got - want) <= 1e-10 * max(1.0, abs(want)), (got, want)


def test_noalloc_rejects_lattices_beyond_the_static_scratch():
    theory = load_theory("Baby Skyrme")
    rp = theory.params.default_params(xlen=16384, ylen=8192, lsx=0.1, lsy=0.1).resolved()  # 131072 tiles
    p_i, p_f = theory.params.pack_device_params(rp)
    f = torch.zeros(8, dtype=torch.float32, device="cuda")  # never read: the size check comes first
    with pytest.raises(ValueError, match="allocation-free"):
        _noalloc_energy(theory.kernels.THEORY_ID, p_i, p_f, "fp32", f)
