"""Reader for the reference's control files (control_MHD, control_sph_shell).

Mirrors the block syntax of the reference's control reader
(F/SERIAL_src/IO/m_read_control_elements.f90, skip_comment_f.f90):

* ``begin NAME`` ... ``end NAME`` nests blocks,
* ``array NAME N`` ... ``end array NAME`` holds N rows of ``NAME v1 v2 ...``,
* ``NAME value`` sets a scalar; ``!`` and ``#`` start comments,
* names compare case-insensitively (cmp_no_case); quoted strings lose quotes.

:func:`shell_params_from_control` turns the subset of keys that the
benchmark configurations use into the parameter set of the time step, with
the equation coefficients built like ``construct_coefficient``
(F/MHD_src/sph_MHD/construct_MHD_coefficient.f90:50-101): the product of
the named dimensionless numbers raised to their powers, where ``One``,
``Two``, ``Zero``, ``Radial_parameter`` and ``Radial_35`` are special names.
Unknown names raise ``ValueError`` as the reference aborts.
"""
from __future__ import annotations

import shlex
from dataclasses import dataclass, field


@dataclass
class Block:
    name: str
    values: dict = field(default_factory=dict)     # lower-case key -> list[str]
    arrays: dict = field(default_factory=dict)     # lower-case key -> list[list[str]]
    blocks: dict = field(default_factory=dict)     # lower-case key -> Block

    def block(self, *path) -> "Block | None":
        b = self
        for p in path:
            b = b.blocks.get(p.lower())
            if b is None:
                return None
        return b

    def get(self, key, default=None):
        v = self.values.get(key.lower())
        return v[0] if v else default

    def array(self, key):
        return self.arrays.get(key.lower(), [])


def _tokens(line: str):
    for c in ("!", "#"):
        i = line.find(c)
        if i >= 0:
            line = line[:i]
    line = line.strip()
    if not line:
        return []
    try:
        return shlex.split(line, posix=True)
    except ValueError:
        return line.split()


def parse_control(text: str) -> Block:
    """Parse a control file into nested :class:`Block` objects."""
    root = Block("root")
    stack = [root]
    arr_name, arr_rows = None, None
    for raw in text.splitlines():
        tok = _tokens(raw)
        if not tok:
            continue
        t0 = tok[0].lower()
        if arr_name is not None:
            if t0 == "end" and len(tok) >= 2 and tok[1].lower() == "array":
                stack[-1].arrays[arr_name] = arr_rows
                arr_name, arr_rows = None, None
            else:
                arr_rows.append(tok[1:])
            continue
        if t0 == "begin" and len(tok) >= 2:
            b = Block(tok[1])
            stack[-1].blocks[tok[1].lower()] = b
            stack.append(b)
        elif t0 == "end":
            if len(stack) == 1:
                raise ValueError(f"unbalanced 'end' in control file: {raw!r}")
            stack.pop()
        elif t0 == "array" and len(tok) >= 2:
            arr_name, arr_rows = tok[1].lower(), []
            if len(tok) >= 3 and tok[2] == "0":
                stack[-1].arrays[arr_name] = []
                arr_name, arr_rows = None, None
        else:
            stack[-1].values[t0] = tok[1:]
    if len(stack) != 1 or arr_name is not None:
        raise ValueError("control file ends inside a block")
    return root


def construct_coefficient(terms, dimless: dict, r_low_t: float, r_high_t: float) -> float:
    """Product of named numbers raised to powers (construct_coefficient)."""
    coef = 1.0
    for row in terms:
        name, power = row[0], float(row[1])
        n = name.lower()
        if n == "one":
            coef = coef * 1.0
        elif n == "two":
            coef = coef * 2.0 ** power
        elif n == "zero":
            coef = coef * 0.0
        elif n == "radial_parameter":
            coef = coef * (1.0 - r_high_t / r_low_t)
        elif n == "radial_35":
            coef = coef * (1.0 - 0.35)
        else:
            if name not in dimless:
                raise ValueError(f"there is missing dimensionless number: {name}")
            coef = coef * dimless[name] ** power
    return coef


def shell_params_from_control(mhd_text: str, shell_text: str, nthreads: int = 0) -> dict:
    """Time-step parameters from control_MHD + control_sph_shell text."""
    mhd = parse_control(mhd_text).block("MHD_control")
    sh = parse_control(shell_text).block("spherical_shell_ctl")
    if mhd is None or sh is None:
        raise ValueError("missing MHD_control or spherical_shell_ctl block")
    g = sh.block("num_grid_sph")
    ltr = int(g.get("truncation_level_ctl"))
    nth = int(g.get("ngrid_meridonal_ctl"))
    nph = int(g.get("ngrid_zonal_ctl"))
    gtype = g.get("radial_grid_type_ctl", "Chebyshev").lower()
    nele = int(g.get("num_fluid_grid_ctl"))
    if g.get("icb_radius_ctl") is not None and g.get("cmb_radius_ctl") is not None:
        r_icb, r_cmb = float(g.get("icb_radius_ctl")), float(g.get("cmb_radius_ctl"))
    else:
        size = float(g.get("fluid_core_size_ctl"))
        ratio = float(g.get("ICB_to_CMB_ratio_ctl"))
        r_icb = size * ratio / (1.0 - ratio)
        r_cmb = r_icb + size
    model = mhd.block("model")
    dimless = {row[0]: float(row[1])
               for row in model.block("dimensionless_ctl").array("dimless_ctl")}
    tdef = model.block("temperature_define")
    use_ref = 0
    dh, dl, ht, lt = r_icb, r_cmb, 1.0, 0.0
    if tdef is not None and (tdef.get("ref_temp_ctl", "none").lower() == "spherical_shell"):
        use_ref = 1
        dl = float(tdef.block("low_temp_ctl").get("depth"))
        lt = float(tdef.block("low_temp_ctl").get("temperature").replace("d", "e"))
        dh = float(tdef.block("high_temp_ctl").get("depth"))
        ht = float(tdef.block("high_temp_ctl").get("temperature").replace("d", "e"))
    coefs = model.block("coefficients_ctl")

    def c(block, arr):
        b = coefs.block(block)
        return construct_coefficient(b.array(arr) if b else [], dimless, dl, dh)

    ctl = mhd.block("control")
    ts = ctl.block("time_step_ctl")
    tl = ctl.block("time_loop_ctl")
    bc = model.block("boundary_condition")
    t_icb, t_cmb = 1.0, 0.0
    for row in bc.array("bc_temperature"):
        if row[1].lower() == "icb":
            t_icb = float(row[2])
        elif row[1].lower() == "cmb":
            t_cmb = float(row[2])
    for row in bc.array("bc_velocity"):
        if row[0].lower() != "non_slip_sph":
            raise ValueError(f"velocity boundary {row[0]} is not supported")
    for row in bc.array("bc_magnetic_field"):
        if row[0].lower() != "insulator":
            raise ValueError(f"magnetic boundary {row[0]} is not supported")
    for row in bc.array("bc_temperature"):
        if row[0].lower() != "fixed":
            raise ValueError(f"thermal boundary {row[0]} is not supported")
    return dict(
        ltr=ltr, nth=nth, nph=nph, nr=nele + 1,
        radial_grid_type=1 if gtype == "chebyshev" else 0,
        r_icb=r_icb, r_cmb=r_cmb,
        dt=float(ts.get("dt_ctl")),
        coef_imp_v=float(tl.get("coef_imp_v_ctl", "0.5")),
        coef_imp_t=float(tl.get("coef_imp_t_ctl", "0.5")),
        coef_imp_b=float(tl.get("coef_imp_b_ctl", "0.5")),
        coef_velo=c("momentum", "coef_4_velocity_ctl"),
        coef_d_velo=c("momentum", "coef_4_v_diffuse_ctl"),
        coef_buo=c("momentum", "coef_4_buoyancy_ctl"),
        coef_cor=c("momentum", "coef_4_Coriolis_ctl"),
        coef_lor=c("momentum", "coef_4_Lorentz_ctl"),
        coef_temp=c("thermal", "coef_4_termal_ctl"),
        coef_d_temp=c("thermal", "coef_4_t_diffuse_ctl"),
        coef_magne=c("induction", "coef_4_magnetic_ctl"),
        coef_d_magne=c("induction", "coef_4_m_diffuse_ctl"),
        coef_induct=c("induction", "coef_4_induction_ctl"),
        use_ref_temp=use_ref, depth_high_t=dh, depth_low_t=dl,
        high_temp=ht, low_temp=lt, temp_icb=t_icb, temp_cmb=t_cmb,
        nthreads=nthreads,
    )


def time_control(mhd_text: str) -> dict:
    """Step counters of time_step_ctl and the loop selectors of time_loop_ctl."""
    ctl = parse_control(mhd_text).block("MHD_control").block("control")
    ts, tl = ctl.block("time_step_ctl"), ctl.block("time_loop_ctl")
    return dict(
        i_step_init=int(ts.get("i_step_init_ctl", "0")),
        i_step_finish=int(ts.get("i_step_finish_ctl", "0")),
        i_step_check=int(ts.get("i_step_check_ctl", "0")),
        i_step_rst=int(ts.get("i_step_rst_ctl", "0")),
        dt=float(ts.get("dt_ctl")),
        legendre_trans_loop=(tl.get("Legendre_trans_loop_ctl") or "").upper(),
        fft_library=(tl.get("FFT_library_ctl") or "").upper(),
    )


def precision_from_control(mhd_text: str) -> int:
    """Precision of the transforms a control_MHD selects through
    Legendre_trans_loop_ctl (set_legendre_trans_mode_ctl,
    legendre_transform_select.f90:181-224): 'B200_mixed' or 'B200_tcgen05'
    -> the mixed path, any other value -> the float64 path.  FFT_library_ctl
    names (set_fft_library_ctl) all select the library's own FFT, in that
    precision."""
    from .sph_mhd import legendre_trans_mode
    return legendre_trans_mode(time_control(mhd_text)["legendre_trans_loop"])
