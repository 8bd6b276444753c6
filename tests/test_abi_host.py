"""The C ABI library loads, exports every function include/soliton_b200.h declares,
and validates its arguments on the host (no kernel launch, no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from soliton_solver_b200 import _native as nat
from soliton_solver_b200.theories import load_theory

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "soliton_b200.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(ss_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = nat.load()
    names = _declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(nat.EXPORTS)
    assert lib.ss_abi_version() == 1


def _prototypes():
    """{name: number of parameters} of every entry point the header declares."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for name, params in re.findall(r"^\s*(?:int|const char \*)\s*(ss_\w+)\s*\(([^)]*)\)\s*;", src, flags=re.M):
        params = params.strip()
        out[name] = 0 if params in ("", "void") else len(params.split(","))
    return out


def test_binding_signatures_match_the_header():
    """The ctypes signature table declares every header entry point with the header's
    number of parameters (a mismatch would pass garbage through the C ABI)."""
    protos = _prototypes()
    assert set(protos) == set(_declared())
    for name, n in protos.items():
        args, _ = nat._SIG[name]
        assert len(args) == n, (name, len(args), n)


def _create(theory_name, **kw):
    th = load_theory(theory_name)
    p_i, p_f = th.params.pack_device_params(th.params.default_params(**kw).resolved())
    h = ctypes.c_void_p()
    rc = nat.load().ss_create(th.kernels.THEORY_ID, p_i.ctypes.data, len(p_i), p_f.ctypes.data, len(p_f),
                              nat.SS_FP32, ctypes.byref(h))
    return rc, h, p_i, p_f


def test_create_and_workspace_size():
    lib = nat.load()
    rc, h, p_i, p_f = _create("Chiral magnet", xlen=100, ylen=70, demag=True)
    assert rc == 0
    n = ctypes.c_size_t()
    assert lib.ss_workspace_bytes(h, ctypes.byref(n)) == 0
    # l1, l2, T4 and stage 4's two accumulated inputs: 5 FP32 field-sized buffers at least
    assert n.value >= 5 * 4 * 4 * 100 * 70
    assert lib.ss_destroy(h) == 0


@pytest.mark.parametrize("mutate,msg", [
    (lambda pi, pf: pi.__setitem__(2, 1), "halo"),
    (lambda pi, pf: pi.__setitem__(4, 3), "number_total_fields"),
    (lambda pi, pf: pi.__setitem__(5, 7), "dim_grid"),
    (lambda pi, pf: pf.__setitem__(2, -1.0), "spacings"),
    (lambda pi, pf: pi.__setitem__(3, 3), "number_coordinates"),
])
def test_create_rejects_bad_params(mutate, msg):
    lib = nat.load()
    th = load_theory("Chiral magnet")
    p_i, p_f = th.params.pack_device_params(th.params.default_params(xlen=20, ylen=20).resolved())
    mutate(p_i, p_f)
    h = ctypes.c_void_p()
    rc = lib.ss_create(0, p_i.ctypes.data, len(p_i), p_f.ctypes.data, len(p_f), nat.SS_FP32, ctypes.byref(h))
    assert rc == nat.SS_ERR_ARG
    assert msg in lib.ss_last_error().decode()
    with pytest.raises(ValueError):
        nat.check(rc)


def test_calls_before_bind_are_rejected():
    lib = nat.load()
    rc, h, _, _ = _create("Baby Skyrme", xlen=16, ylen=16)
    assert rc == 0
    assert lib.ss_step(h, 1, 0.0, None, None) == nat.SS_ERR_STATE
    assert lib.ss_gradient(h, None, None, None) == nat.SS_ERR_STATE
    lib.ss_destroy(h)


def test_short_param_arrays_and_bad_ids():
    lib = nat.load()
    h = ctypes.c_void_p()
    p_i = np.zeros(4, np.int32)
    p_f = np.zeros(4)
    assert lib.ss_create(0, p_i.ctypes.data, 4, p_f.ctypes.data, 4, 1, ctypes.byref(h)) == nat.SS_ERR_ARG
    assert lib.ss_create(9, p_i.ctypes.data, 4, p_f.ctypes.data, 4, 1, ctypes.byref(h)) == nat.SS_ERR_ARG
    assert lib.ss_create(0, p_i.ctypes.data, 4, p_f.ctypes.data, 4, 7, ctypes.byref(h)) == nat.SS_ERR_ARG


def test_render_rgba_validates_arguments_on_the_host():
    """ss_render_rgba rejects bad arguments before launching anything."""
    lib = nat.load()
    buf = ctypes.c_void_p(64)  # never dereferenced: every call below fails validation first
    assert lib.ss_render_rgba(nat.SS_RENDER_JET, None, nat.SS_FP64, 4, 4, 0.0, 1.0, buf, None) == nat.SS_ERR_ARG
    assert lib.ss_render_rgba(7, buf, nat.SS_FP64, 4, 4, 0.0, 1.0, buf, None) == nat.SS_ERR_ARG
    assert lib.ss_render_rgba(nat.SS_RENDER_GRAY, buf, nat.SS_PLAIN_FP64, 4, 4, 0.0, 1.0, buf, None) == nat.SS_ERR_ARG
    assert lib.ss_render_rgba(nat.SS_RENDER_GRAY, buf, nat.SS_FP32, 0, 4, 0.0, 1.0, buf, None) == nat.SS_ERR_ARG
    assert lib.ss_render_rgba(nat.SS_RENDER_GRAY, buf, nat.SS_FP32, 4, 4, 0.0, 1.0, ctypes.c_void_p(66), None) \
        == nat.SS_ERR_ARG
    assert b"aligned" in lib.ss_last_error()


def test_custom_ops_registered_with_fake_shapes():
    """The torch.library ops exist without a GPU, and their fake implementations give
    the output shapes and dtypes (what torch.compile and fake-tensor tracing see)."""
    import torch
    from torch._subclasses.fake_tensor import FakeTensorMode

    from soliton_solver_b200 import autograd as ops  # noqa: F401 (registers the ops)
    for name in ("energy", "energy_gradient", "gradient", "charge", "coupling_grad", "flow_step"):
        assert hasattr(torch.ops.soliton_b200, name)
    with FakeTensorMode():
        f = torch.empty(4 * 8 * 8, dtype=torch.float32)
        v = torch.empty_like(f)
        g = torch.ops.soliton_b200.gradient(f, 1)
        assert g.shape == f.shape and g.dtype == f.dtype
        q = torch.ops.soliton_b200.charge(f, 1, "skyrmion")
        assert q.shape == () and q.dtype == torch.float64
        E, err = torch.ops.soliton_b200.flow_step(f, v, 1, 7, 0.0)
        assert E.shape == (7,) and err.shape == (7,) and E.dtype == torch.float64
