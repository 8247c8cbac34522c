"""The fused Crank-Nicolson kernel against the separate kernels on the GPU.

The time step's explicit update, radial solves and derived fields run either
as one kernel per (field, (l, m) column) (tuning entry TUNE_CN = 1) or as
the separate explicit, implicit and derived kernels (TUNE_CN = 0, the
default; the autotuner times both).  Both evaluate the same
expressions; they may differ only in how the compiler fuses multiply-adds,
so every slot the step writes must agree to rounding, through the Euler
first step and the Adams-Bashforth steps after it."""
import numpy as np
import pytest

from calypso_b200 import PREC_FP64, PREC_MIXED, SphMHD, configs
from calypso_b200.sph_mhd import TUNE_CN

pytestmark = pytest.mark.gpu

# slots the Crank-Nicolson stage writes: velocity, vorticity, magnetic field,
# current density (3 each), temperature, the diffusion terms (3, 3, 1), the
# buoyancy and the previous-step forces (3, 3, 1)
SLOTS = list(range(0, 13)) + list(range(13, 20)) + [47] + list(range(51, 58))


def run(p, prec, fused, steps, seed):
    g = SphMHD(p, prec, device=0)
    t = g.tuning
    assert t[TUNE_CN] in (0, 1), "the fused kernel should take this shell"
    t[TUNE_CN] = fused
    g.tuning = t
    g.init_fields(2, seed)
    g.step(steps)
    out = np.stack([g.get_field(s) for s in SLOTS])
    e = g.energies()
    g.close()
    return out, e


# the small shell's poloidal-velocity operator pivots (the factor form with
# row interchanges), the L63 shell's operators do not (the narrow forms)
SHELLS = {"L31": configs.small_shell(),
          "L63": configs.shell_params(63, 33, 96, 192, E=1e-4, Ra=300.0, dt=5e-6)}


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
@pytest.mark.parametrize("steps", [1, 4])
@pytest.mark.parametrize("shell", sorted(SHELLS))
def test_fused_step_matches_separate_kernels(prec, steps, shell):
    p = SHELLS[shell]
    a, ea = run(p, prec, 1, steps, 7)
    b, eb = run(p, prec, 0, steps, 7)
    for q, s in enumerate(SLOTS):
        scale = max(np.max(np.abs(b[q])), 1e-300)
        err = np.max(np.abs(a[q] - b[q])) / scale
        assert err <= 1e-12, (s, err)
    assert np.allclose(ea, eb, rtol=1e-12, atol=0.0)


def test_fused_step_at_the_benchmark_shape():
    # L = 255, 129 radial levels: the poloidal velocity and poloidal magnetic
    # operators pivot at every degree (both forms with row interchanges)
    p = configs.full_step_L255()
    a, ea = run(p, PREC_FP64, 1, 2, 3)
    b, eb = run(p, PREC_FP64, 0, 2, 3)
    for q, s in enumerate(SLOTS):
        scale = max(np.max(np.abs(b[q])), 1e-300)
        assert np.max(np.abs(a[q] - b[q])) / scale <= 1e-12, s
    assert np.allclose(ea, eb, rtol=1e-12, atol=0.0)


def test_autotune_times_both_and_the_choice_sticks():
    p = configs.small_shell()
    g = SphMHD(p, PREC_FP64, device=0)
    t = g.autotune()
    assert t[TUNE_CN] in (0, 1)
    g.tuning = [4, 2, 2, 384, 1 - t[TUNE_CN]]
    assert g.tuning[TUNE_CN] == 1 - t[TUNE_CN]
    g.close()
