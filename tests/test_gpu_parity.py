"""GPU parity of the float64 plain path against the CPU oracle and the
reference's golden energies.  Tolerances: Gauss nodes / P_l^m 1e-13, SHT
1e-12 relative L2, time-stepped fields 1e-10 relative L2, golden energies
1e-9 (the reference's own regression tolerance); config 0's full 2000-step
run: energies and spectra 1e-9 (float64) and 1e-6 (mixed path)."""
import json
import os

import numpy as np
import pytest

from calypso_b200 import PREC_FP64, PREC_MIXED, SphMHD, configs
from calypso_b200.sph_mhd import CURRENT, MAGNE, TEMP, VELO, VORT

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dynamobench_case1")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def random_spec(L, nr, nc, seed, zero_l0_dpol=(), zero_l0=()):
    rng = np.random.default_rng(seed)
    jmax = (L + 1) ** 2
    ls = np.array([l for l in range(L + 1) for _ in range(2 * l + 1)])
    amp = 1.0 / np.sqrt(2 * ls + 1.0) / np.maximum(ls, 1)
    spec = rng.standard_normal((nc, nr, jmax)) * amp[None, None, :]
    for c in zero_l0:
        spec[c, :, 0] = 0.0
    return spec


@pytest.fixture(scope="module")
def case1():
    return configs.dynamobench_case1()


def test_tables_match_oracle(oracle_lib, case1):
    g = SphMHD(case1, PREC_FP64)
    o = oracle_lib.Oracle(case1)
    c1, w1 = g.gauss()
    c2, w2 = o.gauss()
    assert np.abs(c1 - c2).max() < 1e-14
    assert np.abs(w1 - w2).max() < 1e-14
    for l, m in [(0, 0), (1, 0), (5, 3), (20, 7), (31, 0), (31, 1), (31, 31)]:
        p1, d1 = g.plm(l, m)
        p2, d2 = o.plm(l, m)
        s = max(np.abs(p2).max(), 1e-300)
        assert np.abs(p1 - p2).max() / s < 1e-13, (l, m)
        sd = max(np.abs(d2).max(), 1e-300)
        assert np.abs(d1 - d2).max() / sd < 1e-12, (l, m)


# float64 Legendre kernels (tuning entries 0 and 1): on the CUDA cores
# (backward 4, forward 2) and on the float64 tensor cores (1, 3)
KERNELS = {"cuda_cores": [4, 2], "tensor_cores": [1, 3]}


@pytest.mark.parametrize("kern", sorted(KERNELS))
@pytest.mark.parametrize("nvec,nscal", [(3, 2), (4, 1), (1, 0), (0, 1), (2, 6)])
def test_sht_fp64_matches_oracle(oracle_lib, case1, nvec, nscal, kern):
    g = SphMHD(case1, PREC_FP64)
    g.tuning = KERNELS[kern]
    o = oracle_lib.Oracle(case1)
    nc = 3 * nvec + nscal
    zl0 = [3 * v + 1 for v in range(nvec)] + [3 * v + 2 for v in range(nvec)]
    spec = random_spec(g.L, g.nr, nc, 7 + nc, zero_l0=zl0)
    grid_g = g.sph_back_trans(nvec, nscal, spec)
    grid_o = o.sht_backward(nvec, nscal, spec)
    for c in range(nc):
        assert rel_l2(grid_g[c], grid_o[c]) < 1e-12, c
    back_g = g.sph_forward_trans(nvec, nscal, grid_o)
    back_o = o.sht_forward(nvec, nscal, grid_o)
    for c in range(nc):
        assert rel_l2(back_g[c], back_o[c]) < 1e-12, c
        # round trip is the identity for band-limited data
        assert rel_l2(back_g[c], spec[c]) < 1e-11, c


def test_dynamobench_case1_golden_energies(case1):
    with open(os.path.join(GOLD, "sph_pwr_volume_s.json")) as f:
        gold = json.load(f)
    g = SphMHD(case1, PREC_FP64)
    g.init_fields(1)
    for row in gold["rows"]:
        g.step(row["step"] - g.istep)
        e = g.energies()
        ref = np.array(row["values"])
        rel = np.abs(e - ref) / np.abs(ref)
        assert rel.max() <= gold["rel_tol"], (row["step"], rel)


def test_fp64_kernels_L127_match_oracle(oracle_lib):
    """L127, 192 Gauss nodes (96 per hemisphere: one full and one partial
    64-node tile of the tensor-core backward kernel; two 64-degree blocks,
    the second partial, of the forward one), Nr 9 (a partial radial tile),
    4 vectors + 1 scalar: both pairs of float64 Legendre kernels against the
    oracle, backward and forward, 1e-12 relative L2 per component."""
    p = configs.shell_params(127, 9, 192, 384, E=1e-4, Ra=300.0, dt=5e-6)
    o = oracle_lib.Oracle(dict(p, nthreads=os.cpu_count() or 1))
    nvec, nscal = 4, 1
    nc = 3 * nvec + nscal
    zl0 = [3 * v + 1 for v in range(nvec)] + [3 * v + 2 for v in range(nvec)]
    spec = random_spec(127, 9, nc, 21, zero_l0=zl0)
    grid_o = o.sht_backward(nvec, nscal, spec)
    back_o = o.sht_forward(nvec, nscal, grid_o)
    for kern in sorted(KERNELS):
        g = SphMHD(p, PREC_FP64)
        g.tuning = KERNELS[kern]
        grid_g = g.sph_back_trans(nvec, nscal, spec)
        back_g = g.sph_forward_trans(nvec, nscal, grid_o)
        g.close()
        for c in range(nc):
            assert rel_l2(grid_g[c], grid_o[c]) < 1e-12, (kern, c, rel_l2(grid_g[c], grid_o[c]))
            assert rel_l2(back_g[c], back_o[c]) < 1e-12, (kern, c, rel_l2(back_g[c], back_o[c]))


def _compare_fields(g, o, tol):
    for slot in (VELO, VELO + 1, VELO + 2, VORT, VORT + 2, MAGNE, MAGNE + 1, MAGNE + 2,
                 CURRENT, CURRENT + 2, TEMP):
        a, b = g.get_field(slot), o.get_field(slot)
        assert rel_l2(a, b) < tol, (slot, rel_l2(a, b))


@pytest.mark.parametrize("kern", sorted(KERNELS))
def test_case1_fields_match_oracle(oracle_lib, case1, kern):
    g = SphMHD(case1, PREC_FP64)
    g.tuning = KERNELS[kern]
    o = oracle_lib.Oracle(case1)
    g.init_fields(1)
    o.init_fields(1)
    _compare_fields(g, o, 1e-10)
    g.step(20)
    o.step(20)
    _compare_fields(g, o, 1e-10)
    np.testing.assert_allclose(g.energies(), o.energies(), rtol=1e-11)


def test_small_shell_seeded_matches_oracle(oracle_lib):
    p = configs.small_shell()
    g = SphMHD(p, PREC_FP64)
    o = oracle_lib.Oracle(p)
    g.init_fields(2, seed=3)
    o.init_fields(2, 3)
    _compare_fields(g, o, 1e-10)
    g.step(400)
    o.step(400)
    _compare_fields(g, o, 1e-10)
    np.testing.assert_allclose(g.energies(), o.energies(), rtol=1e-10)


def test_graph_replay_is_bitwise_eager(case1):
    a = SphMHD(case1, PREC_FP64)
    b = SphMHD(case1, PREC_FP64)
    a.init_fields(1)
    b.init_fields(1)
    a.step(12)
    b.step(12, graph=True)
    for slot in (VELO, MAGNE + 2, TEMP):
        assert np.array_equal(a.get_field(slot), b.get_field(slot)), slot


def test_host_state_step_matches_device_step(case1):
    slots = [3, 5, 13, 15, 48, 50, 51, 53, 6, 8, 16, 18, 38, 40, 54, 56, 12, 19, 41, 57]
    a = SphMHD(case1, PREC_FP64)
    a.init_fields(1)
    a.step(5)
    state = np.stack([a.get_field(s) for s in slots])
    a.step(1)
    b = SphMHD(case1, PREC_FP64)
    b.init_fields(1)
    b.step_host_state(state)
    for q, s in enumerate(slots):
        np.testing.assert_allclose(state[q], a.get_field(s), rtol=0, atol=1e-12 * np.abs(a.get_field(s)).max() + 1e-300)


def test_energy_spectra_match_oracle(oracle_lib, case1):
    """Volume spectra by l, |m| and l - |m| (sph_pwr_volume_l/_m/_lm.dat)
    after 20 steps of case 1: 1e-10 relative to each spectrum's total; each
    spectrum sums to the volume energies."""
    g = SphMHD(case1, PREC_FP64)
    o = oracle_lib.Oracle(case1)
    g.init_fields(1)
    o.init_fields(1)
    g.step(20)
    o.step(20)
    sg, so = g.energy_spectra(), o.energy_spectra()
    e = g.energies()
    for kind in ("l", "m", "lm"):
        a, b = sg[kind], so[kind]
        for q in range(7):
            tot = np.abs(b[q]).sum()
            assert np.abs(a[q] - b[q]).max() <= 1e-10 * tot, (kind, q)
            assert abs(a[q].sum() - e[q]) <= 1e-12 * abs(e[q]), (kind, q)


def test_bench_shell_fp64_matches_oracle(oracle_lib):
    """The bench workload itself (L255, Nr129, 384 x 768, seeded start):
    the float64 path against the oracle after the Euler step and one
    Adams-Bashforth step, 1e-10 relative L2 per field."""
    p = configs.full_step_L255()
    g = SphMHD(p, PREC_FP64)
    o = oracle_lib.Oracle(dict(p, nthreads=os.cpu_count() or 1))
    g.init_fields(2, seed=1)
    o.init_fields(2, 1)
    g.step(2)
    o.step(2)
    _compare_fields(g, o, 1e-10)
    np.testing.assert_allclose(g.energies(), o.energies(), rtol=1e-10)


def test_config0_full_run_energies_and_spectra(oracle_lib):
    """Config 0 as stated: L31, Nr33, 48 x 96, E 1e-3, Ra 100, seeded start,
    dt 1e-4, 2000 steps, energies and spectra against the oracle.  float64
    path: energies 1e-9 relative, spectra 1e-9 of each spectrum's total
    (2000 steps of differently ordered float64 sums); mixed path: energies
    1e-6, spectra 1e-6 of each spectrum's total."""
    import os
    p = configs.small_shell()
    o = oracle_lib.Oracle(dict(p, nthreads=os.cpu_count() or 1))
    o.init_fields(2, 5)
    o.step(2000)
    eo, so = o.energies(), o.energy_spectra()
    for prec, tol in ((PREC_FP64, 1e-9), (PREC_MIXED, 1e-6)):
        g = SphMHD(p, prec)
        g.init_fields(2, seed=5)
        g.step(1)
        g.step(1999, graph=True)
        eg, sg = g.energies(), g.energy_spectra()
        g.close()
        np.testing.assert_allclose(eg, eo, rtol=tol)
        for kind in ("l", "m", "lm"):
            for q in range(7):
                tot = np.abs(so[kind][q]).sum()
                assert np.abs(sg[kind][q] - so[kind][q]).max() <= tol * tot, (prec, kind, q)
