"""Learned spectral subgrid closure: host side (cb2_mlp_* / cb2_closure_*).

The training data comes from the solver itself: a high-resolution shell is
advanced, each snapshot is filtered onto the low-resolution shell
(cb2_filter_fields: l <= L_lo, every stride-th Chebyshev point), and the
target is the filtered high-resolution nonlinear terms minus the terms the
low-resolution solver computes from the filtered state.  The network is
trained on the GPU by the library's own forward / backward / Adam kernels;
torch tensors only hold the device buffers.  The plain low-resolution
solver is the fallback (detach the closure) and, against the filtered
high-resolution run, the yardstick of the closure's error.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from .sph_mhd import CalypsoError, SphMHD, _check, load_library

NIN, NOUT = 16, 5
OUT_SLOTS = (48, 50, 38, 40, 41)      # curl of forces S, T; induction S, T; heat advection


def _lib():
    L = load_library()
    P, vp, i, f32, d = ctypes.POINTER, ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
    sig = {
        "cb2_mlp_create": ([i, i, i, ctypes.c_uint, P(vp)], i),
        "cb2_mlp_destroy": ([vp], i),
        "cb2_mlp_num_params": ([vp], i),
        "cb2_mlp_get_params": ([vp, P(f32)], i),
        "cb2_mlp_set_params": ([vp, P(f32)], i),
        "cb2_mlp_forward": ([vp, vp, ctypes.c_longlong, vp], i),
        "cb2_mlp_loss_grad": ([vp, vp, vp, ctypes.c_longlong, P(d), P(f32)], i),
        "cb2_mlp_adam_step": ([vp, f32, f32, f32, f32], i),
        "cb2_mlp_sync": ([vp], i),
        "cb2_filter_fields": ([vp, vp], i),
        "cb2_filter_terms": ([vp, vp, vp], i),
        "cb2_closure_features": ([vp, vp], i),
        "cb2_closure_targets": ([vp, vp, vp], i),
        "cb2_closure_attach": ([vp, vp, P(f32)], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


def _fptr(a: np.ndarray):
    if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
        raise CalypsoError("float32 C-contiguous array expected")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dev(t):
    """device pointer of a contiguous torch CUDA tensor"""
    if not t.is_cuda or not t.is_contiguous():
        raise CalypsoError("contiguous CUDA tensor expected")
    return ctypes.c_void_p(t.data_ptr())


class MLP:
    """nin -> nhid -> nhid -> nout network on the GPU (bfloat16 weights)."""

    def __init__(self, nin: int = NIN, nhid: int = 256, nout: int = NOUT, seed: int = 0):
        lib = _lib()
        h = ctypes.c_void_p()
        _check(lib.cb2_mlp_create(nin, nhid, nout, seed, ctypes.byref(h)), "cb2_mlp_create")
        self._h = h
        self.nin, self.nhid, self.nout = nin, nhid, nout
        self.nparams = lib.cb2_mlp_num_params(h)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib().cb2_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparams, np.float32)
        _check(_lib().cb2_mlp_get_params(self._h, _fptr(out)), "cb2_mlp_get_params")
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        _check(_lib().cb2_mlp_set_params(self._h, _fptr(p)), "cb2_mlp_set_params")

    def forward(self, x):
        import torch
        torch.cuda.synchronize()
        y = torch.empty((x.shape[0], self.nout), device=x.device, dtype=torch.float32)
        _check(_lib().cb2_mlp_forward(self._h, _dev(x), x.shape[0], _dev(y)), "cb2_mlp_forward")
        return y

    def loss_grad(self, x, t, want_grad: bool = False):
        import torch
        torch.cuda.synchronize()
        loss = ctypes.c_double()
        g = np.zeros(self.nparams, np.float32) if want_grad else None
        _check(_lib().cb2_mlp_loss_grad(self._h, _dev(x), _dev(t), x.shape[0], ctypes.byref(loss),
                                        _fptr(g) if want_grad else None), "cb2_mlp_loss_grad")
        return (loss.value, g) if want_grad else loss.value

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        _check(_lib().cb2_mlp_adam_step(self._h, lr, beta1, beta2, eps), "cb2_mlp_adam_step")

    def sync(self):
        _check(_lib().cb2_mlp_sync(self._h), "cb2_mlp_sync")


def filter_fields(src: SphMHD, dst: SphMHD):
    _check(_lib().cb2_filter_fields(src._h, dst._h), "cb2_filter_fields")


def snapshot_pair(hi: SphMHD, lo: SphMHD):
    """features and targets (torch CUDA float32) of the current hi state on lo"""
    import torch
    n = lo.nr * lo.jmax
    filter_fields(hi, lo)
    terms = torch.empty((NOUT, n), device="cuda", dtype=torch.float64)
    _check(_lib().cb2_filter_terms(hi._h, lo._h, _dev(terms)), "cb2_filter_terms")
    x = torch.empty((n, NIN), device="cuda", dtype=torch.float32)
    y = torch.empty((n, NOUT), device="cuda", dtype=torch.float32)
    _check(_lib().cb2_closure_features(lo._h, _dev(x)), "cb2_closure_features")
    _check(_lib().cb2_closure_targets(lo._h, _dev(terms), _dev(y)), "cb2_closure_targets")
    return x, y


def generate(hi: SphMHD, lo: SphMHD, n_snap: int, every: int):
    """n_snap (features, targets) pairs, hi advanced `every` steps between them"""
    xs, ys = [], []
    for _ in range(n_snap):
        hi.step(every, graph=True)
        x, y = snapshot_pair(hi, lo)
        xs.append(x)
        ys.append(y)
    return xs, ys


class Normaliser:
    """Per radial level k: mean / std of each field feature (the geometry
    features l/L, m/L, r stay as they are) and std of each target.  The two
    wall levels carry no closure: they are left out of training."""

    def __init__(self, xs, ys, nr: int):
        import torch
        self.nr = nr
        x = torch.stack(xs).view(len(xs), nr, -1, NIN)
        y = torch.stack(ys).view(len(ys), nr, -1, NOUT)
        self.jmax = x.shape[2]
        self.mean = x.mean((0, 2))
        self.std = x.std((0, 2)).clamp_min(1e-30)
        self.mean[:, 13:] = 0.0
        self.std[:, 13:] = 1.0
        self.yscale = y.std((0, 2)).clamp_min(1e-30)
        self.yscale[0] = 1.0
        self.yscale[-1] = 1.0

    def x(self, x):
        v = x.view(self.nr, self.jmax, NIN)
        return ((v - self.mean[:, None, :]) / self.std[:, None, :]).reshape(-1, NIN).contiguous()

    def y(self, y):
        v = y.view(self.nr, self.jmax, NOUT)
        return (v / self.yscale[:, None, :]).reshape(-1, NOUT).contiguous()

    def interior(self, a):
        """rows of the interior radial levels 1 .. nr-2"""
        return a[self.jmax:(self.nr - 1) * self.jmax]

    def host_norm(self, alpha: float = 1.0) -> np.ndarray:
        return np.concatenate([self.mean.cpu().numpy().ravel(), self.std.cpu().numpy().ravel(),
                               (alpha * self.yscale).cpu().numpy().ravel()]).astype(np.float32)


def train(net: MLP, xs, ys, norm: Normaliser, epochs: int = 2, batch: int = 16384, lr: float = 1e-3, seed: int = 0):
    """minibatch Adam over the interior rows of all snapshots; mean loss per epoch"""
    import torch
    x = torch.cat([norm.interior(norm.x(a)) for a in xs])
    y = torch.cat([norm.interior(norm.y(b)) for b in ys])
    n = x.shape[0]
    batch = min(batch, n)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    hist = []
    for _ in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        tot, cnt = 0.0, 0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            xb, yb = x[idx].contiguous(), y[idx].contiguous()
            tot += net.loss_grad(xb, yb)
            cnt += 1
            net.adam_step(lr)
        hist.append(tot / max(cnt, 1))
    net.sync()
    return hist


def explained(net: MLP, norm: Normaliser, xs, ys) -> float:
    """1 - |tau - tau_pred|^2 / |tau|^2 over the interior rows (normalised units)"""
    num = den = 0.0
    for x, y in zip(xs, ys):
        yn = norm.interior(norm.y(y))
        p = norm.interior(net.forward(norm.x(x)))
        num += float(((p - yn) ** 2).sum())
        den += float((yn ** 2).sum())
    return 1.0 - num / den


def attach(ctx: SphMHD, net: MLP | None, norm: Normaliser | None = None, alpha: float = 1.0):
    """attach the closure (tendency scaled by alpha), or detach it (net None)"""
    if net is None:
        _check(_lib().cb2_closure_attach(ctx._h, None, None), "cb2_closure_attach")
        return
    hn = norm.host_norm(alpha)
    _check(_lib().cb2_closure_attach(ctx._h, net._h, _fptr(hn)), "cb2_closure_attach")


def energy_spectra(ctx: SphMHD) -> np.ndarray:
    """kinetic and magnetic energy per degree l (2 x (L+1)), trapezoid in r"""
    L, nr = ctx.L, ctx.nr
    r = _radii(ctx)
    j = np.arange((L + 1) ** 2)
    l = np.floor(np.sqrt(j)).astype(int)
    g = l * (l + 1.0)
    w = np.zeros(nr)
    w[1:] += 0.5 * np.diff(r)
    w[:-1] += 0.5 * np.diff(r)
    out = np.zeros((2, L + 1))
    for q, base in enumerate((0, 6)):
        S, dS, T = (ctx.get_field(base + c) for c in range(3))
        e = g / (2 * l + 1.0) * (g * S ** 2 / r[:, None] ** 2 + dS ** 2 + T ** 2) * 0.5
        e[:, 0] = 0.0
        out[q] = np.bincount(l, weights=(w[:, None] * e).sum(0), minlength=L + 1)
    return out


def _radii(ctx: SphMHD) -> np.ndarray:
    p = ctx.params
    ri, ro, nr = p["r_icb"], p["r_cmb"], p["nr"]
    if p.get("radial_grid_type", 1) == 1:
        return np.array([ri + 0.5 * (ro - ri) * (1.0 - math.cos(math.pi * k / (nr - 1))) for k in range(nr)])
    return np.linspace(ri, ro, nr)


def spectra_error(a: np.ndarray, b: np.ndarray) -> float:
    """relative L2 distance of two spectra (both kinetic and magnetic)"""
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
