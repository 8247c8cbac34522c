"""Named workloads: the shells the benchmark configurations describe.

Every configuration uses the physics family of the reference's dynamo
benchmark control file (tests/Dynamobench_case1/control_MHD): Boussinesq
MHD in a shell with r_i/r_o = 0.35 and fluid_core_size 1, non-slip
isothermal walls, insulating magnetic boundaries, the spherical-shell
reference temperature, and the coefficients

    c_buo = (1 - 0.35) Ra / E,  c_cor = 2 / E,  c_lor = 1 / (Pm E),
    c_dT = 1 / Pr,  c_dB = 1 / Pm,  c_v = c_dv = c_T = c_B = c_ind = 1.
"""
from __future__ import annotations

RATIO = 0.35


def shell_params(L: int, nr: int, nth: int, nph: int, E: float, Ra: float,
                 Pr: float = 1.0, Pm: float = 5.0, dt: float = 1e-4,
                 coef_imp: float = 0.6, radial_grid_type: int = 1) -> dict:
    r_icb = 1.0 * RATIO / (1.0 - RATIO)
    r_cmb = r_icb + 1.0
    return dict(
        ltr=L, nth=nth, nph=nph, nr=nr, radial_grid_type=radial_grid_type,
        r_icb=r_icb, r_cmb=r_cmb, dt=dt,
        coef_imp_v=coef_imp, coef_imp_t=coef_imp, coef_imp_b=coef_imp,
        coef_velo=1.0, coef_d_velo=1.0, coef_buo=(1.0 - RATIO) * Ra / E,
        coef_cor=2.0 / E, coef_lor=1.0 / (Pm * E),
        coef_temp=1.0, coef_d_temp=1.0 / Pr,
        coef_magne=1.0, coef_d_magne=1.0 / Pm, coef_induct=1.0,
        use_ref_temp=1, depth_high_t=r_icb, depth_low_t=r_cmb,
        high_temp=1.0, low_temp=0.0, temp_icb=1.0, temp_cmb=0.0, nthreads=0,
    )


def dynamobench_case1() -> dict:
    """tests/Dynamobench_case1: L31, 49 Chebyshev points, E 1e-3, Ra 100, dt 5e-5."""
    p = shell_params(31, 49, 48, 96, E=1e-3, Ra=100.0, dt=5e-5)
    p.update(depth_high_t=0.5384615384615384, depth_low_t=1.5384615384615384)
    return p


def small_shell() -> dict:
    """Plain FP64 small case: L31, Nr33, E 1e-3, Ra 100, dt 1e-4 (2000 steps)."""
    return shell_params(31, 33, 48, 96, E=1e-3, Ra=100.0, dt=1e-4)


def sht_roundtrip() -> dict:
    """Isolated SHT round trip: L255, 384 Gauss nodes, 768 longitudes, Nr65."""
    return shell_params(255, 65, 384, 768, E=1e-4, Ra=300.0, dt=5e-6)


def sht_roundtrip_spectra(L: int, nr: int, nvec: int = 3, nscal: int = 2):
    """Seeded spectra of the SHT round-trip workload: field f (the vectors,
    then the scalars) draws from seed f independent N(0, 1) values for every
    real harmonic coefficient (the cos and sin parts of m are separate
    coefficients), scaled by 1 / (l sqrt(2l+1)) so that the power of degree
    l, summed over m, falls as l^-2 (l = 0 scaled as l = 1).  A vector's
    three slots (S, dS/dr, T) come from the same stream; its dS/dr and T
    have no l = 0 part.  Array (3 nvec + nscal, nr, (L+1)^2), j = l(l+1)+m."""
    import numpy as np
    ls = np.array([l for l in range(L + 1) for _ in range(2 * l + 1)])
    amp = 1.0 / (np.maximum(ls, 1) * np.sqrt(2 * ls + 1.0))
    out = []
    for f in range(nvec + nscal):
        rng = np.random.default_rng(f)
        ncomp = 3 if f < nvec else 1
        x = rng.standard_normal((ncomp, nr, (L + 1) ** 2)) * amp[None, None, :]
        if f < nvec:
            x[1:, :, 0] = 0.0
        out.append(x)
    return np.concatenate(out)


def full_step_L255() -> dict:
    """Full time step: L255, Nr129, 384 x 768 grid, E 1e-4, Ra 300.

    dt = 5e-6 is fixed here for both precision paths: the Coriolis term is
    explicit (Adams-Bashforth) with coefficient 2/E = 2e4, and
    2/E * dt = 0.1 is the value of the reference's own benchmark case
    (2e3 * 5e-5)."""
    return shell_params(255, 129, 384, 768, E=1e-4, Ra=300.0, dt=5e-6)


CONFIGS = {
    "dynamobench_case1": dynamobench_case1,
    "small_shell_L31_Nr33": small_shell,
    "sht_roundtrip_L255_Nr65": sht_roundtrip,
    "full_step_L255_Nr129": full_step_L255,
}


ENSEMBLE_SHAPES = (
    # (L, Nr, Ntheta, Nphi, dt): Ntheta = 3(L+1)/2 and Nphi = 2 Ntheta as in the
    # reference's L31 grid; dt halves with each doubling of L
    (31, 33, 48, 96, 1e-4),
    (63, 65, 96, 192, 5e-5),
    (127, 97, 192, 384, 2.5e-5),
)


def ensemble(n_per_shape: int = 16, seed: int = 0, E: float = 1e-3, ra_range=(80.0, 400.0)) -> list:
    """Batched ensemble: n_per_shape shells of each of ENSEMBLE_SHAPES, the
    physics of the small shell with the Rayleigh number of each shell drawn
    uniformly in ra_range (seeded).  48 shells by default."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for (L, nr, nth, nph, dt) in ENSEMBLE_SHAPES:
        for _ in range(n_per_shape):
            ra = float(rng.uniform(*ra_range))
            out.append(shell_params(L, nr, nth, nph, E=E, Ra=ra, dt=dt))
    return out
