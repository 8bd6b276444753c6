"""Initial-condition hooks with the reference's names, run by libsoliton_b200.

``make_initial_config(theory_id, key)`` returns, for one theory, the functions of
``soliton_solver/theories/<theory>/initial_config.py`` on the native kernels
(``ss_initialize`` / ``ss_insert_soliton``):

* ``initialize(*, Velocity, Field, ..., config)``: ``mode`` "ground" (also "uniform",
  "vacuum", "gs") or "initial" (the default, as in the reference): the soliton ansatz
  at the lattice centre.  Config keys as the reference's: ``ansatz`` ("bloch", "neel",
  "anti"; default "bloch") and ``skyrmion_rotation`` for the chiral magnet and baby
  Skyrme, ``vortex_number`` (default 1) for the Abelian Higgs model.  The reference's
  chiral-magnet and baby-Skyrme "initial" path passes one argument too few and cannot
  run; this one does.  The caller's RK4 scratch buffers (k1..l4, Temp) are zeroed.
* ``create_ground_state_kernel[grid, block](Velocity, Field, grid, k1, .., Temp, p_i, p_f)``,
  ``create_initial_configuration_kernel[grid, block](...)`` (the theory's own argument
  list), ``create_skyrmion_kernel[grid, block](Field, grid, pxi, pxj, skyrmion_rotation,
  ansatz_bloch, ansatz_neel, ansatz_anti, p_i, p_f)`` (chiral magnet, baby Skyrme) and
  ``create_vortex_kernel[grid, block](Field, grid, pxi, pxj, vortex, p_i, p_f)`` (Abelian
  Higgs, s+id).  The launch configuration and the coordinate grid are accepted and not
  needed (coordinates are lsx * x, lsy * y, as create_grid_kernel writes them).
"""
from __future__ import annotations

from soliton_solver_b200 import _native as nat
from soliton_solver_b200.core.hooks import Launch, as_tensor
from soliton_solver_b200.core.solver import solver_for

_ANSATZ = {"bloch": nat.SS_ANSATZ_BLOCH, "neel": nat.SS_ANSATZ_NEEL, "anti": nat.SS_ANSATZ_ANTI}
_MAGNETIC = ("chiral_magnet", "baby_skyrme")


def _flags_to_ansatz(bloch, neel, anti):
    if bloch:
        return nat.SS_ANSATZ_BLOCH
    if neel:
        return nat.SS_ANSATZ_NEEL
    if anti:
        return nat.SS_ANSATZ_ANTI
    return nat.SS_ANSATZ_NONE


def make_initial_config(theory_id: int, key: str) -> dict:
    def _init(Velocity, Field, p_i, p_f, mode, ansatz=nat.SS_ANSATZ_BLOCH, rotation=0.0, vortex_number=1.0,
              scratch=()):
        v = as_tensor(Velocity) if Velocity is not None else None
        f = as_tensor(Field)
        s = solver_for(theory_id, p_i, p_f, f.dtype, f.device)
        s.initialize(f, v, mode, ansatz, rotation, vortex_number)
        for buf in scratch:
            if buf is not None:
                as_tensor(buf).zero_()

    def initialize(*, Velocity, Field, grid=None, k1=None, k2=None, k3=None, k4=None, l1=None, l2=None, l3=None,
                   l4=None, Temp=None, p_i_d=None, p_f_d=None, p_i_h=None, p_f_h=None, grid2d=None, block2d=None,
                   config: dict | None = None, rp=None):
        cfg = config or {}
        p_i = p_i_h if p_i_h is not None else p_i_d
        p_f = p_f_h if p_f_h is not None else p_f_d
        if p_i is None or p_f is None:
            raise ValueError("initialize needs the packed parameters (p_i_h/p_f_h or p_i_d/p_f_d)")
        scratch = (k1, k2, k3, k4, l1, l2, l3, l4, Temp)
        mode = str(cfg.get("mode", "initial")).lower()
        if mode in ("ground", "uniform", "vacuum", "gs"):
            _init(Velocity, Field, p_i, p_f, nat.SS_INIT_GROUND, scratch=scratch)
            return
        ansatz = _ANSATZ.get(str(cfg.get("ansatz", "bloch")).lower(), nat.SS_ANSATZ_BLOCH)
        _init(Velocity, Field, p_i, p_f, nat.SS_INIT_ANSATZ, ansatz, float(cfg.get("skyrmion_rotation", 0.0)),
              float(cfg.get("vortex_number", 1.0)), scratch)

    def create_ground_state_kernel(Velocity, Field, grid, k1, k2, k3, k4, l1, l2, l3, l4, Temp, p_i, p_f):
        _init(Velocity, Field, p_i, p_f, nat.SS_INIT_GROUND, scratch=(k1, k2, k3, k4, l1, l2, l3, l4, Temp))

    out = {"initialize": initialize,
           "create_ground_state_kernel": Launch(create_ground_state_kernel, "create_ground_state_kernel")}

    if key in _MAGNETIC:
        def create_initial_configuration_kernel(Velocity, Field, grid, k1, k2, k3, k4, l1, l2, l3, l4, Temp,
                                                ansatz_bloch, ansatz_neel, ansatz_anti, skyrmion_rotation,
                                                vortex_number, p_i, p_f):
            _init(Velocity, Field, p_i, p_f, nat.SS_INIT_ANSATZ, _flags_to_ansatz(ansatz_bloch, ansatz_neel,
                                                                                  ansatz_anti),
                  float(skyrmion_rotation), 1.0, (k1, k2, k3, k4, l1, l2, l3, l4, Temp))

        def create_skyrmion_kernel(Field, grid, pxi, pxj, skyrmion_rotation, ansatz_bloch, ansatz_neel, ansatz_anti,
                                   p_i, p_f):
            f = as_tensor(Field)
            s = solver_for(theory_id, p_i, p_f, f.dtype, f.device)
            s.insert_soliton(f, int(pxi), int(pxj), _flags_to_ansatz(ansatz_bloch, ansatz_neel, ansatz_anti), 0,
                             float(skyrmion_rotation))

        out["create_skyrmion_kernel"] = Launch(create_skyrmion_kernel, "create_skyrmion_kernel")
    else:
        if key == "ginzburg_landau_superconductor":
            def create_initial_configuration_kernel(Velocity, Field, grid, k1, k2, k3, k4, l1, l2, l3, l4, Temp,
                                                    vortex_number, p_i, p_f):
                _init(Velocity, Field, p_i, p_f, nat.SS_INIT_ANSATZ, nat.SS_ANSATZ_NONE, 0.0, float(vortex_number),
                      (k1, k2, k3, k4, l1, l2, l3, l4, Temp))
        else:
            def create_initial_configuration_kernel(Velocity, Field, grid, k1, k2, k3, k4, l1, l2, l3, l4, Temp,
                                                    p_i, p_f):
                _init(Velocity, Field, p_i, p_f, nat.SS_INIT_ANSATZ, nat.SS_ANSATZ_NONE, 0.0, 1.0,
                      (k1, k2, k3, k4, l1, l2, l3, l4, Temp))

        def create_vortex_kernel(Field, grid, pxi, pxj, vortex, p_i, p_f):
            f = as_tensor(Field)
            s = solver_for(theory_id, p_i, p_f, f.dtype, f.device)
            s.insert_soliton(f, int(pxi), int(pxj), nat.SS_ANSATZ_NONE, 1 if vortex else 0, 0.0)

        out["create_vortex_kernel"] = Launch(create_vortex_kernel, "create_vortex_kernel")
    out["create_initial_configuration_kernel"] = Launch(create_initial_configuration_kernel,
                                                        "create_initial_configuration_kernel")
    return out
