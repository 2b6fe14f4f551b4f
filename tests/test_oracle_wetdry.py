"""The oracle under WETDRY (-DWETDRY; hydrodynamic_module.f90:510-570,
interpolation_module.f90:628-939, 1022-1136): frame masks equal to the
static masks change nothing; a cell dry in every slot has no velocity."""
import ctypes as C

import numpy as np

import harness
from oracle import oracle as O
from romspath_b200 import schedule


def test_static_masks_as_frame_masks_change_nothing():
    case = harness.make_case("tiny", 200, seed=3, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    ref, _ = harness.run_oracle(case, 36)
    g = case.grid
    masks = {"wetdry_rho": g["mask_rho"].astype(np.float64), "wetdry_u": g["mask_u"].astype(np.float64),
             "wetdry_v": g["mask_v"].astype(np.float64)}
    case2 = harness.make_case("tiny", 200, seed=3, spec_over={"diag": True},
                              param_over={**harness.DIAG_PARAMS, "wetdry": 1})
    orig = case2.frame

    def frame(k, ng=1):
        f = dict(orig(k, ng))
        f.update(masks)
        return f
    case2.frame = frame
    got, _ = harness.run_oracle(case2, 36)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_dry_cell_has_no_velocity():
    case = harness.make_case("tiny", 10, seed=3, spec_over={"wetdry": True}, param_over={"wetdry": 1})
    m = O.OracleModel(case.specs, case.grids, case.params)
    f = dict(case.stored(1))
    wr = case.grid["mask_rho"].astype(np.float64).copy()
    wr[9:13, 8:12] = 0.0            # a dry patch around rho points (10..13, 9..12)
    f["wetdry_rho"] = wr
    f["wetdry_u"] = wr[:-1, :] * wr[1:, :]
    f["wetdry_v"] = wr[:, :-1] * wr[:, 1:]
    for slot in (1, 2, 3):
        m.set_frame(1, slot, f)
    fl = C.c_uint32(0)
    # the centre of the patch: every u, v corner of the cell is dry
    for var in (0, 1):              # ORC_V_U, ORC_V_V
        val = O.lib().orc_getinterp3d(C.byref(m.g[0]), var, 11.5, 10.5, -5.0, 1, 1, 0.0, -30.0, C.byref(fl))
        assert val == 0.0
    # outside the patch the same call sees the current
    for var in (0, 1):
        val = O.lib().orc_getinterp3d(C.byref(m.g[0]), var, 16.5, 14.5, -5.0, 1, 1, 0.0, -30.0, C.byref(fl))
        assert val != 0.0


def test_frames_carry_time_varying_masks():
    case = harness.make_case("tiny", 10, seed=3, spec_over={"wetdry": True}, param_over={"wetdry": 1})
    dry = [int((case.grid["mask_rho"] - case.frame(k)["wetdry_rho"]).sum()) for k in range(1, 13)]
    assert max(dry) > 10 and min(dry) == 0
