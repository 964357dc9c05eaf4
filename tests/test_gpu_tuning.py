"""Tuning knobs and the autotuner change speed, never results.

The candidate-row skin only changes which non-overlapping partners a row
carries and how often rows are rebuilt; the pass-kernel variant only changes
the register budget of the same code; the launch shape (block size,
particles per thread, pair grid, persistent chunks) only how the same code
is launched.  Trajectories must stay bit-identical."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem

pytestmark = pytest.mark.gpu


def _system(precision):
    pos, rad, L = configs.relaxed_tile(3000, 0.55, 17, relax_steps=100)
    vel = np.random.default_rng(3).normal(0.0, 0.3, (len(rad), 3))
    s = DEMSystem(configs.dense_packing_params(0.6, L, precision=precision))
    s.set_state(pos, vel, np.zeros_like(vel), radius=rad)
    s.initialize_cell_distribution()
    return s


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_MIXED])
def test_autotune_keeps_the_trajectory(precision):
    a, b = _system(precision), _system(precision)
    a.run(1, 8)
    t = a.autotune(9, 4)
    assert t["last_step"] == 8 + DEMSystem.AUTOTUNE_TRIALS * 8
    assert t["skin_factor"] in (0.025, 0.05, 0.1) and t["pass_variant"] in (0, 1, 2)
    assert t["particles_per_thread"] in (1, 2, 4) and t["test_block"] in (64, 128, 256)
    assert t["pair_waves"] in (1, 2, 4) and t["launch_mode"] in (0, 1)
    assert all(ms > 0 for ms in t["trial_ms"])  # (the persistent trial ran too)
    b.run(1, t["last_step"])
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    ca, cb = a.get_contacts(), b.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert a.ncol() == b.ncol()


def test_tuning_settings_keep_the_trajectory():
    ref = _system(P.PREC_FP64)
    ref.run(1, 40)
    want = ref.get_state()
    for skin, variant in ((0.01, 1), (0.2, 0), (0.1, 1), (0.05, 2)):
        s = _system(P.PREC_FP64)
        s.set_tuning(skin, variant)
        s.run(1, 40)
        got = s.get_state()
        for k in want:
            np.testing.assert_array_equal(got[k], want[k], err_msg=f"{skin} {variant} {k}")


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_MIXED])
def test_early_launch_keeps_the_trajectory(precision):
    """Test, pair and fold kernels launched with programmatic stream
    serialization (the default) against plain stream order: the same bits,
    in graph-replayed chunks and in passes launched one by one."""
    a, b = _system(precision), _system(precision)
    assert a.early_launch()
    b.set_early_launch(False)
    assert not b.early_launch()
    for s in (a, b):
        s.run(1, 60)
        for k in range(61, 66):
            s.move_particles(k)
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    ca, cb = a.get_contacts(), b.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert a.ncol() == b.ncol()
