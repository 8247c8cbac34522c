"""Batched ensemble and kernel-variant autotuner on the GPU.

  - every shell of an ensemble (mixed truncations, one CUDA graph launch per
    step) ends bit-for-bit where the same shell stepped alone ends, with the
    mixed path's Legendre GEMMs as one launch over all shells or one per
    shell;
  - the autotuner picks from its candidate sets, refuses to run once the
    fields exist, and no kernel variant changes a result (bitwise)."""
import numpy as np
import pytest

from calypso_b200 import PREC_FP64, PREC_MIXED, CalypsoError, Ensemble, SphMHD, configs
from calypso_b200.sph_mhd import MAGNE, TEMP, VELO

pytestmark = pytest.mark.gpu

CANDIDATES = [(1, 2, 4), (1, 2, 3), (1, 2, 4), (384, 512, 256, 128)]


def small_ensemble():
    out = []
    for q, (L, nr, nth, nph, dt) in enumerate([(31, 17, 48, 96, 1e-4), (63, 17, 96, 192, 5e-5)]):
        for ra in (120.0, 300.0):
            out.append(configs.shell_params(L, nr, nth, nph, E=1e-3, Ra=ra, dt=dt))
    return out


@pytest.mark.parametrize("prec,batched", [(PREC_MIXED, True), (PREC_MIXED, False), (PREC_FP64, True)])
def test_ensemble_matches_shells_stepped_alone(prec, batched):
    params = small_ensemble()
    ens = Ensemble(params, prec, device=0, autotune=True)
    ens.set_batched(batched)
    ens.init_fields(2, 11)
    ens.step(12)
    e_ens = ens.energies()
    fields = [[s.get_field(slot) for slot in (VELO, MAGNE + 2, TEMP)] for s in ens.shells]
    tunings = [s.tuning for s in ens.shells]
    ens.close()
    for q, p in enumerate(params):
        g = SphMHD(p, prec, device=0)
        g.tuning = tunings[q]
        g.init_fields(2, 11 + q)
        g.step(12, graph=True)
        assert np.array_equal(g.energies(), e_ens[q]), q
        for a, slot in zip(fields[q], (VELO, MAGNE + 2, TEMP)):
            assert np.array_equal(a, g.get_field(slot)), (q, slot)
        g.close()


def test_batched_legendre_launches_three_truncations():
    """Mixed shells of three truncations in an unsorted order (L31, L127,
    L63, L31: different colatitude counts, B-table heights and tensor-memory
    widths in one launch) and four radial sizes: the ensemble whose two
    Legendre GEMMs are one launch over every shell's tiles ends bitwise where
    the ensemble with one launch per shell ends, and switching between the
    two forms in the middle of a run changes nothing."""
    params = [configs.shell_params(31, 9, 48, 96, E=1e-3, Ra=150.0, dt=1e-4),
              configs.shell_params(127, 9, 192, 384, E=1e-4, Ra=300.0, dt=5e-6),
              configs.shell_params(63, 13, 96, 192, E=1e-3, Ra=250.0, dt=5e-5),
              configs.shell_params(31, 17, 48, 96, E=1e-3, Ra=350.0, dt=1e-4)]
    runs = []
    for mode in ("batched", "branches", "switch"):
        ens = Ensemble(params, PREC_MIXED, device=0, autotune=False)
        ens.set_batched(mode != "branches")
        ens.init_fields(2, 5)
        ens.step(4)
        if mode == "switch":
            ens.set_batched(False)
        ens.step(4)
        runs.append((ens.energies(), [[s.get_field(slot) for slot in (VELO, MAGNE + 2, TEMP)]
                                      for s in ens.shells]))
        ens.close()
    for e, f in runs[1:]:
        assert np.array_equal(e, runs[0][0])
        for q in range(len(params)):
            for a, b in zip(f[q], runs[0][1][q]):
                assert np.array_equal(a, b), q
    assert np.isfinite(runs[0][0]).all()


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_FP64])
def test_autotune_candidates_and_state(prec):
    p = configs.small_shell()
    g = SphMHD(p, prec, device=0)
    t = g.autotune()
    for q, cand in enumerate(CANDIDATES):
        assert t[q] in cand or q in ((2, 3) if prec == PREC_FP64 else (0, 1)), (q, t)
    g.init_fields(2, 3)
    with pytest.raises(CalypsoError):
        g.autotune()
    g.close()


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_FP64])
def test_kernel_variants_give_identical_results(prec):
    p = configs.small_shell()
    ref = None
    variants = [[2, 1, 1, 128], [4, 2, 2, 256], [2, 2, 4, 512]]
    for v in variants:
        g = SphMHD(p, prec, device=0)
        g.tuning = v
        g.init_fields(2, 5)
        g.step(6)
        f = np.stack([g.get_field(s) for s in (VELO, MAGNE, TEMP)])
        g.close()
        if ref is None:
            ref = f
        else:
            assert np.array_equal(f, ref), v


def test_small_shell_created_after_large_one_leaves_it_working():
    # kernel shared-memory limits are process-wide: a small shell must not
    # lower them below what a larger shell created earlier launches with
    big = configs.shell_params(63, 33, 96, 192, E=1e-4, Ra=300.0, dt=5e-6)
    small = configs.shell_params(31, 17, 48, 96, E=1e-4, Ra=300.0, dt=5e-6)
    for prec in (PREC_MIXED, PREC_FP64):
        a = SphMHD(big, prec, device=0)
        b = SphMHD(small, prec, device=0)
        a.init_fields(2, 1)
        b.init_fields(2, 1)
        a.step(3)
        b.step(3)
        assert np.all(np.isfinite(a.energies())) and np.all(np.isfinite(b.energies()))
        a.close()
        b.close()


@pytest.mark.parametrize("prec,tol", [(PREC_MIXED, 1e-5), (PREC_FP64, 1e-12)])
def test_four_step_and_stockham_fft_agree(prec, tol):
    # tuning value 384 runs the four-step products kernel (nphi = 3 (L + 1)),
    # 512 the Stockham kernel: the same transform up to rounding, in float32
    # (mixed path) and in float64 (plain path)
    p = configs.small_shell()
    assert p["nph"] == 3 * (p["ltr"] + 1)
    out = []
    for nt in (384, 512):
        g = SphMHD(p, prec, device=0)
        t = g.tuning
        t[3] = nt
        g.tuning = t
        g.init_fields(2, 5)
        g.step(6)
        out.append(np.stack([g.get_field(s) for s in (VELO, MAGNE, TEMP)]))
        g.close()
    for a, b in zip(out[0], out[1]):
        assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b)
