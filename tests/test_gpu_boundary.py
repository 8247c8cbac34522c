"""Routine-level entry points on the reference's rlm / rtm / rtp buffers
(cb2_leg_bwd / cb2_leg_fwd = sel_backward/forward_legendre_trans,
cb2_fft_bwd / cb2_fft_fwd = back/fwd_MHD_FFT_sel_from_recv, cb2_fft_products
= the grid products with the FFTs around them) against the oracle's halves
of the transform, on index tables with permuted modes and non-trivial
strides.

Tolerances (relative L2 per component): float64 context 1e-12 (the same
sums in another order); mixed context 5e-6 for the Legendre transforms (the
split-fp16 products, see test_gpu_mixed.py) and 2e-6 for the float32 FFT
and products (float32 transforms, each pair of rows scaled to its own
size)."""
import ctypes

import numpy as np
import pytest

from calypso_b200 import PREC_FP64, PREC_MIXED, CalypsoError, SphMHD, configs, load_library, sph_tables
from calypso_b200.sph_mhd import rlm_size, rtm_size

pytestmark = pytest.mark.gpu

TOL_LEG = {PREC_FP64: 1e-12, PREC_MIXED: 5e-6}
TOL_FFT = {PREC_FP64: 1e-12, PREC_MIXED: 2e-6}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def tables_for(p, seed, permuted=True):
    """Tables with the modes in a seeded random order, k running fastest in
    rlm, the orders fastest in rtm and theta fastest in rtp."""
    L, nr, nth, nph = p["ltr"], p["nr"], p["nth"], p["nph"]
    rng = np.random.default_rng(seed)
    jo = [(l, m) for l in range(L + 1) for m in range(-l, l + 1)]
    mo = list(range(-L, L + 1))
    if permuted:
        jo = [jo[i] for i in rng.permutation(len(jo))]
        mo = [mo[i] for i in rng.permutation(len(mo))]
    nj, nm = len(jo), len(mo)
    return sph_tables(L, nr, nth, nph, j_order=jo, m_order=mo, istep_rlm=(1, nr),
                      istep_rtm=(nm, nm * nr, 1), istep_rtp=(nth, 1, nth * nr))


def spec_to_rlm(spec, t, ncomp):
    """[c][k][j = l(l+1)+m] -> sp_rlm(comp + ncomp ((k-1) istep(1) + (j-1) istep(2)))"""
    nc, nr, _ = spec.shape
    WR = np.zeros(rlm_size(t, ncomp))
    jg = np.array([l * (l + 1) + m for (l, m) in t.j_order])
    k = np.arange(nr)
    for c in range(nc):
        idx = c + ncomp * (k[:, None] * t.istep_rlm[0] + np.arange(len(jg))[None, :] * t.istep_rlm[1])
        WR[idx] = spec[c][:, jg]
    return WR


def rlm_to_spec(WS, t, ncomp, nc, jmax):
    nr = t.nidx_rlm[0]
    spec = np.zeros((nc, nr, jmax))
    jg = np.array([l * (l + 1) + m for (l, m) in t.j_order])
    k = np.arange(nr)
    for c in range(nc):
        idx = c + ncomp * (k[:, None] * t.istep_rlm[0] + np.arange(len(jg))[None, :] * t.istep_rlm[1])
        spec[c][:, jg] = WS[idx]
    return spec


def four_to_rtm(four, t, ncomp):
    """oracle Fourier array [c][k][theta][m + L] -> vr_rtm"""
    nc, nr, nth, ns = four.shape
    L = (ns - 1) // 2
    WR = np.zeros(rtm_size(t, ncomp))
    k, th = np.arange(nr), np.arange(nth)
    for q, m in enumerate(t.m_order):
        base = k[:, None] * t.istep_rtm[0] + th[None, :] * t.istep_rtm[1] + q * t.istep_rtm[2]
        for c in range(nc):
            WR[c + ncomp * base] = four[c, :, :, m + L]
    return WR


def rtm_to_four(WS, t, ncomp, nc, L):
    nr, nth = t.nidx_rtm[0], t.nidx_rtm[1]
    four = np.zeros((nc, nr, nth, 2 * L + 1))
    k, th = np.arange(nr), np.arange(nth)
    for q, m in enumerate(t.m_order):
        base = k[:, None] * t.istep_rtm[0] + th[None, :] * t.istep_rtm[1] + q * t.istep_rtm[2]
        for c in range(nc):
            four[c, :, :, m + L] = WS[c + ncomp * base]
    return four


def rtp_to_grid(F, t, nc):
    nr, nth, nph = t.nidx_rtp[0], t.nidx_rtp[1], t.nidx_rtp[2]
    nnod = nr * nth * nph
    k, th, ph = np.meshgrid(np.arange(nr), np.arange(nth), np.arange(nph), indexing="ij")
    inod = k * t.istep_rtp[0] + th * t.istep_rtp[1] + ph * t.istep_rtp[2]
    return np.stack([F[c * nnod + inod] for c in range(nc)])


def grid_to_rtp(g, t):
    nc, nr, nth, nph = g.shape
    nnod = nr * nth * nph
    F = np.zeros(nnod * nc)
    k, th, ph = np.meshgrid(np.arange(nr), np.arange(nth), np.arange(nph), indexing="ij")
    inod = k * t.istep_rtp[0] + th * t.istep_rtp[1] + ph * t.istep_rtp[2]
    for c in range(nc):
        F[c * nnod + inod] = g[c]
    return F


def random_spec(L, nr, nc, seed, nvec):
    rng = np.random.default_rng(seed)
    ls = np.array([l for l in range(L + 1) for _ in range(2 * l + 1)])
    amp = 1.0 / np.sqrt(2 * ls + 1.0) / np.maximum(ls, 1)
    spec = rng.standard_normal((nc, nr, (L + 1) ** 2)) * amp[None, None, :]
    for v in range(nvec):          # no l = 0 part of dS/dr and T
        spec[3 * v + 1, :, 0] = 0.0
        spec[3 * v + 2, :, 0] = 0.0
    return spec


def random_four(L, nr, nth, nc, seed, scales=None):
    rng = np.random.default_rng(seed)
    four = rng.standard_normal((nc, nr, nth, 2 * L + 1)) / np.sqrt(1.0 + np.abs(np.arange(-L, L + 1)))
    if scales is not None:
        four *= np.asarray(scales)[:, None, None, None]
    return four


PRECS = [PREC_FP64, PREC_MIXED]


@pytest.fixture(scope="module")
def case1():
    return configs.dynamobench_case1()


@pytest.mark.parametrize("prec", PRECS)
def test_legendre_only_matches_oracle(oracle_lib, case1, prec):
    g = SphMHD(case1, prec)
    o = oracle_lib.Oracle(case1)
    t = tables_for(case1, 5)
    nvec, nscal = 3, 2
    nc = 3 * nvec + nscal
    ncomp = nc + 1                    # one component the call must leave alone
    spec = random_spec(g.L, g.nr, nc, 17, nvec)
    WR = spec_to_rlm(spec, t, ncomp)
    WS = g.sel_backward_legendre_trans(ncomp, nvec, nscal, WR, t)
    four = rtm_to_four(WS, t, ncomp, nc, g.L)
    four_o = o.leg_backward(nvec, nscal, spec)
    for c in range(nc):
        assert rel_l2(four[c], four_o[c]) < TOL_LEG[prec], (c, rel_l2(four[c], four_o[c]))
    # forward: the oracle's Fourier coefficients back to spectra
    WR2 = four_to_rtm(four_o, t, ncomp)
    WS2 = g.sel_forward_legendre_trans(ncomp, nvec, nscal, WR2, t)
    back = rlm_to_spec(WS2, t, ncomp, nc, g.jmax)
    back_o = o.leg_forward(nvec, nscal, four_o)
    for c in range(nc):
        assert rel_l2(back[c], back_o[c]) < TOL_LEG[prec], (c, rel_l2(back[c], back_o[c]))
    # the Legendre transforms are exact for band-limited data
    for c in range(nc):
        assert rel_l2(back_o[c], spec[c]) < 1e-11, c


@pytest.mark.parametrize("prec", PRECS)
def test_fft_only_matches_oracle(oracle_lib, case1, prec):
    g = SphMHD(case1, prec)
    o = oracle_lib.Oracle(case1)
    t = tables_for(case1, 6)
    nc = 15                            # more than one chunk of 13
    four = random_four(g.L, g.nr, g.nth, nc, 21, scales=np.logspace(-3, 2, nc))
    WR = four_to_rtm(four, t, nc)
    F = g.back_MHD_FFT_sel_from_recv(nc, WR, t)
    grid = rtp_to_grid(F, t, nc)
    grid_o = o.fft_backward(four)
    for c in range(nc):
        assert rel_l2(grid[c], grid_o[c]) < TOL_FFT[prec], (c, rel_l2(grid[c], grid_o[c]))
    WS = g.fwd_MHD_FFT_sel_from_recv(nc, grid_to_rtp(grid_o, t), t)
    four_b = rtm_to_four(WS, t, nc, nc, g.L)
    four_bo = o.fft_forward(grid_o)
    for c in range(nc):
        assert rel_l2(four_b[c], four_bo[c]) < TOL_FFT[prec], (c, rel_l2(four_b[c], four_bo[c]))


@pytest.mark.parametrize("prec", PRECS)
def test_legendre_then_fft_is_the_whole_transform(case1, prec):
    g = SphMHD(case1, prec)
    t = tables_for(case1, 7, permuted=False)
    nvec, nscal = 4, 1
    nc = 13
    spec = random_spec(g.L, g.nr, nc, 23, nvec)
    WS = g.sel_backward_legendre_trans(nc, nvec, nscal, spec_to_rlm(spec, t, nc), t)
    grid = rtp_to_grid(g.back_MHD_FFT_sel_from_recv(nc, WS, t), t, nc)
    whole = g.sph_back_trans(nvec, nscal, spec)
    for c in range(nc):
        assert rel_l2(grid[c], whole[c]) < 1e-13, c


def np_fft_backward(four, nph):
    """[c][k][theta][m + L] -> grid [c][k][theta][phi]: f = a_0 + sum (a_m cos + b_m sin),
    each component transformed on its own (numpy, float64)."""
    L = (four.shape[-1] - 1) // 2
    F = np.zeros(four.shape[:-1] + (nph // 2 + 1,), dtype=complex)
    F[..., 0] = four[..., L]
    for m in range(1, L + 1):
        F[..., m] = 0.5 * (four[..., L + m] - 1j * four[..., L - m])
    return np.fft.irfft(F, n=nph, axis=-1) * nph


def np_fft_forward(grid, L):
    """grid [c][k][theta][phi] -> [c][k][theta][m + L] (a_0 = mean, a_m, b_m = 2/N sums)."""
    nph = grid.shape[-1]
    F = np.fft.rfft(grid, axis=-1) / nph
    four = np.zeros(grid.shape[:-1] + (2 * L + 1,))
    four[..., L] = F[..., 0].real
    for m in range(1, L + 1):
        four[..., L + m] = 2 * F[..., m].real
        four[..., L - m] = -2 * F[..., m].imag
    return four


def _products(grid, cv, cl, ci, ct):
    u, w, B, J, T = grid[0:3], grid[3:6], grid[6:9], grid[9:12], grid[12]

    def cross(a, b):
        return np.stack([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])
    return np.concatenate([cv * cross(w, u), cl * cross(J, B), ci * cross(u, B), ct * u * T[None]])


# field sizes: velocity, vorticity, magnetic field, current density,
# temperature.  "skewed" (a weak field beside an order-one flow) puts rows of
# very different size into one complex transform; the float64 kernel scales
# each pair to one size and meets 1e-12 on it.  The float32 step kernels
# pair rows of related size without scaling and are checked on "balanced"
# sizes (within a factor 30, as in the bench state).
SKEWED = [1.0, 1.0, 1.0, 30.0, 30.0, 30.0, 1e-4, 1e-4, 1e-4, 3e-3, 3e-3, 3e-3, 0.1]
BALANCED = [1.0, 1.0, 1.0, 10.0, 10.0, 10.0, 0.3, 0.3, 0.3, 3.0, 3.0, 3.0, 0.1]


@pytest.mark.parametrize("prec,fft_threads,scales", [(PREC_FP64, None, SKEWED), (PREC_FP64, None, BALANCED),
                                                     (PREC_MIXED, 384, BALANCED), (PREC_MIXED, 256, BALANCED)])
def test_fft_products_match_fp64_restatement(oracle_lib, case1, prec, fft_threads, scales):
    """The products kernel of the step against float64 FFTs of each
    component on its own and numpy products."""
    g = SphMHD(case1, prec)
    if fft_threads:
        g.tuning = [4, 2, 2, fft_threads, 0]
    o = oracle_lib.Oracle(case1)
    t = tables_for(case1, 8)
    four = random_four(g.L, g.nr, g.nth, 13, 31, scales=scales)
    WS = g.fft_products(four_to_rtm(four, t, 13), t)
    got = rtm_to_four(WS, t, 12, 12, g.L)
    p = case1
    # the reference transforms every component on its own (FFTPACK's
    # multiple real sequences): numpy's float64 FFTs stand in for it here
    grid = np_fft_backward(four, g.nph)
    assert rel_l2(grid, o.fft_backward(four)) < 1e-12
    prod = _products(grid, p["coef_velo"], p["coef_lor"], p["coef_induct"], p["coef_temp"])
    want = np_fft_forward(prod, g.L)
    for c in range(12):
        assert rel_l2(got[c], want[c]) < TOL_FFT[prec], (c, rel_l2(got[c], want[c]))


def test_device_buffers_are_used_in_place(case1):
    import torch
    g = SphMHD(case1, PREC_FP64, device=0)
    t = tables_for(case1, 9)
    nvec, nscal = 1, 1
    nc = 4
    spec = random_spec(g.L, g.nr, nc, 41, nvec)
    WR = spec_to_rlm(spec, t, nc)
    host = g.sel_backward_legendre_trans(nc, nvec, nscal, WR, t)
    dwr = torch.from_numpy(WR).to("cuda:0")
    dws = torch.zeros(rtm_size(t, nc), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    g.sel_backward_legendre_trans(nc, nvec, nscal, dwr.data_ptr(), t, WS=dws.data_ptr())
    assert np.array_equal(dws.cpu().numpy(), host)


def test_routine_entry_points_reject_bad_arguments(case1):
    g = SphMHD(case1, PREC_FP64)
    t = tables_for(case1, 10, permuted=False)
    nc = 3
    WR = np.zeros(rlm_size(t, nc))
    lib = load_library()
    out = np.zeros(rtm_size(t, nc))
    pd = ctypes.c_void_p
    # n_WR one short of the tables' extent
    rc = lib.cb2_leg_bwd(g._h, ctypes.byref(t), nc, 1, 0, WR.size - 1, out.size, pd(WR.ctypes.data),
                         pd(out.ctypes.data))
    assert rc == -1 and b"smaller than" in lib.cb2_last_error()
    # ncomp below 3 nvector + nscalar
    with pytest.raises(CalypsoError):
        g.sel_backward_legendre_trans(2, 1, 0, WR, t)
    # a degree beyond the truncation in the rlm table
    bad = sph_tables(g.L, g.nr, g.nth, g.nph, j_order=[(g.L + 1, 0)] + t.j_order[1:])
    with pytest.raises(CalypsoError):
        g.sel_backward_legendre_trans(nc, 1, 0, np.zeros(rlm_size(bad, nc)), bad)
    # wrong number of colatitudes in the rtm table
    t.nidx_rtm[1] = g.nth - 2
    with pytest.raises(CalypsoError):
        g.back_MHD_FFT_sel_from_recv(nc, np.zeros(rtm_size(t, nc)), t)
