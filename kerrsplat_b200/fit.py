"""The fit-loop side of the render path, on the GPU entry points: the time-resolved visibility
likelihood and its gradient, the matrix-free Gauss-Newton products J v and J^T w in residual space,
LSQR on them, the Levenberg-Marquardt polish, and the device value-and-gradient of the image-domain
chi^2 that Fit.fit!(...; gradient = :dual) takes, with an Adam step on the host.

Restates src/Fit/timeresolved.jl:109-138 (timeresolved_gradient!, device branch),
src/Fit/device_visibilities.jl:14-50 (FrameScans, gains), src/Fit/gauss_newton.jl:45-154 (residuals!,
jvp!, jtvp!), 165-180 (normal_diagonal!), 326-357 (lsqr_step!), 361-412 (polish_timeresolved!) and
src/Fit/Fit.jl:380-434 (fit!'s _dual_valgrad). Every image, transform, seed and sweep runs on the GPU
(ks_render, ks_jvp, ks_adjoint, ks_visibilities, ks_vis_seed, ks_vis_chi2_gradient); what stays on
the host is what the reference keeps there: the per-frame bookkeeping, the LSQR recurrences (FP64)
and the optimiser's step.

Residual layout (gauss_newton.jl:67-85): bands in order, each band's frame times sorted, each
frame's baselines in order, 8 values per baseline: Re and Im of the gained, noise-weighted residual
(g V - d) / sigma of Stokes I, Q, U, V.
"""
import numpy as np

from . import (KS_FP64, KS_MIXED, PolarizedSplats, adjoint, capture_chi2_gradient, chi2_gradient, jvp as image_jvp, render,
               vis_chi2_gradient, vis_seed, visibilities)

__all__ = ["FrameScans", "BandScans", "timeresolved_gradient", "residuals", "jvp", "jtvp", "normal_diagonal", "lsqr", "lsqr_step",
           "polish_timeresolved", "dual_valgrad", "GraphValgrad", "Adam", "fit"]


class FrameScans:
    """The visibility scans of one frame (FrameScans, device_visibilities.jl:14-50): baselines u, v
    (wavelengths), data vis (nuv, 4) complex Jy, noise sigma (nuv, 4), the scattering taper tap
    (ones without a kernel) and the gain factor g = g_s1 conj(g_s2) of every baseline (ones without
    gains)."""

    def __init__(self, u, v, vis, sigma, tap=None, g=None):
        self.u = np.ascontiguousarray(u, dtype=np.float64)
        self.v = np.ascontiguousarray(v, dtype=np.float64)
        n = self.u.size
        self.vis = np.ascontiguousarray(vis, dtype=np.complex128).reshape(n, 4)
        self.sigma = np.ascontiguousarray(np.broadcast_to(sigma, (n, 4)), dtype=np.float64)
        self.tap = None if tap is None else np.ascontiguousarray(tap, dtype=np.float64)
        self.g = np.ones(n, dtype=np.complex128) if g is None else np.ascontiguousarray(g, dtype=np.complex128)
        if self.v.size != n or self.g.size != n or (self.tap is not None and self.tap.size != n):
            raise ValueError("baseline arrays of one frame must have the same length")
        if not np.all(self.sigma > 0):
            raise ValueError("sigma must be positive")

    @property
    def nres(self):
        """8 residual entries per baseline (_nres, gauss_newton.jl:65)."""
        return 8 * self.u.size

    @staticmethod
    def gain_factors(gains, s1, s2):
        """g_s1 conj(g_s2) from a 2 x stations matrix of log-amplitude and phase (ScanGains,
        timeresolved.jl:43-56)."""
        gains = np.asarray(gains, dtype=np.float64)
        gc = np.exp(gains[0] + 1j * gains[1])
        return gc[np.asarray(s1)] * np.conj(gc[np.asarray(s2)])


class BandScans:
    """One frequency's time-resolved scans (BandScans / TimeResolved): frame time -> FrameScans, the
    frequency nu and the transform's pixel size psize (rad) and flux scale (pixel solid angle / Jy)."""

    def __init__(self, frames, nu, psize, scale):
        self.frames = {float(t): fs for t, fs in frames.items()}
        self.times = np.array(sorted(self.frames))
        self.nu = float(nu)
        self.psize = float(psize)
        self.scale = float(scale)

    @property
    def nres(self):
        return sum(self.frames[t].nres for t in self.times)


def _bands(bands):
    return [bands] if isinstance(bands, BandScans) else list(bands)


def residual_length(bands):
    return sum(b.nres for b in _bands(bands))


def _flat(res):
    """(nuv, 4) complex -> 8 reals per baseline: Re I, Im I, Re Q, Im Q, ..."""
    return np.stack([res.real, res.imag], axis=-1).reshape(-1)


def _unflat(x, n):
    y = np.asarray(x, dtype=np.float64).reshape(n, 4, 2)
    return y[..., 0] + 1j * y[..., 1]


def timeresolved_gradient(cache, params, bands, L, precision=KS_MIXED, nmax=-1, slab=0.0):
    """chi^2 of the splat movie against time-resolved visibility scans and its gradient
    (timeresolved_gradient!'s device branch, timeresolved.jl:109-138): one ks_vis_chi2_gradient per
    frame time of every band (forward image, transform, chi^2 and seed, reverse sweep), the gradient
    accumulated in place. Returns (chi2, grad (21, nsplat))."""
    model = PolarizedSplats(params)
    g = np.zeros(np.asarray(params).size)
    total = 0.0
    for b in _bands(bands):
        for t in b.times:
            fs = b.frames[t]
            x, _ = vis_chi2_gradient(cache, model, t, b.nu, L, fs.u, fs.v, fs.vis, fs.sigma, b.psize, b.scale, tap=fs.tap, gains=fs.g,
                                     nmax=nmax, slab=slab, precision=precision, dparams=g)
            total += x
    return total, g.reshape(np.asarray(params).shape[1], -1).T.copy()


def residuals(cache, params, bands, L, precision=KS_MIXED, nmax=-1, slab=0.0):
    """The weighted residuals of every band, frame and baseline (residuals!, gauss_newton.jl:45-63)
    and chi^2 = |r|^2: each band's frames rendered in one call, each frame's transform on the GPU."""
    model = PolarizedSplats(params)
    out = []
    for b in _bands(bands):
        imgs = np.asarray(render(cache, model, b.times, [b.nu], L, nmax=nmax, slab=slab, precision=precision))[0]
        for f, t in enumerate(b.times):
            fs = b.frames[t]
            V = visibilities(cache, imgs[f], fs.u, fs.v, b.psize, b.scale, tap=fs.tap, precision=precision)
            out.append(_flat((fs.g[:, None] * V - fs.vis) / fs.sigma))
    r = np.concatenate(out) if out else np.zeros(0)
    return r, float(r @ r)


def jvp(cache, params, bands, L, dirs, precision=KS_MIXED, nmax=-1, slab=0.0):
    """J v in residual space (jvp!, gauss_newton.jl:91-118) for one direction (21, nsplat) or a
    stack (ndir, 21, nsplat): the image's directional derivatives on the GPU (ks_jvp, duals along
    v), then each frame's transform of them, gained and weighted. Returns (m,) or (ndir, m)."""
    model = PolarizedSplats(params)
    d = np.asarray(dirs, dtype=np.float64)
    one = d.ndim == 2
    d = d[None] if one else d
    out = np.zeros((d.shape[0], residual_length(bands)))
    off = 0
    for b in _bands(bands):
        dimg = image_jvp(cache, model, b.times, [b.nu], L, d, nmax=nmax, slab=slab, precision=precision)   # (ndir, 1, nt, npix, 4)
        for f, t in enumerate(b.times):
            fs = b.frames[t]
            n = fs.nres
            for k in range(d.shape[0]):
                dV = visibilities(cache, dimg[k, 0, f], fs.u, fs.v, b.psize, b.scale, tap=fs.tap, precision=precision)
                out[k, off:off + n] = _flat(fs.g[:, None] * dV / fs.sigma)
            off += n
    return out[0] if one else out


def jtvp(cache, params, bands, L, w, precision=KS_MIXED, nmax=-1, slab=0.0):
    """J^T w in parameter space (jtvp!, gauss_newton.jl:126-154): every frame's adjoint transform of
    conj(g) w / sigma (ks_vis_seed) seeds one reverse sweep over the band's frames (ks_adjoint).
    Returns (21, nsplat)."""
    params = np.asarray(params, dtype=np.float64)
    model = PolarizedSplats(params)
    w = np.asarray(w, dtype=np.float64)
    if w.size != residual_length(bands):
        raise ValueError(f"w must have {residual_length(bands)} entries, got {w.size}")
    g = np.zeros(params.size)
    off = 0
    for b in _bands(bands):
        seeds = np.zeros((1, b.times.size, cache.npix, 4))
        for f, t in enumerate(b.times):
            fs = b.frames[t]
            n = fs.nres
            wc = np.conj(fs.g)[:, None] * _unflat(w[off:off + n], fs.u.size) / fs.sigma
            seeds[0, f] = vis_seed(cache, wc, fs.u, fs.v, b.psize, b.scale, tap=fs.tap, precision=precision)
            off += n
        adjoint(cache, model, b.times, [b.nu], L, seeds, nmax=nmax, slab=slab, precision=precision, dparams=g)
    return g.reshape(params.shape[1], -1).T.copy()


def normal_diagonal(cache, params, bands, L, probes=8, rng=None, mask=None, precision=KS_MIXED, nmax=-1, slab=0.0):
    """Hutchinson estimate of diag(J^T J) (normal_diagonal!, gauss_newton.jl:165-180): the mean of
    z * J^T (J z) over Rademacher probes z, in absolute value, floored at 1e-6 of its largest entry."""
    rng = np.random.default_rng() if rng is None else rng
    params = np.asarray(params, dtype=np.float64)
    dg = np.zeros_like(params)
    for _ in range(max(int(probes), 1)):
        z = rng.choice([-1.0, 1.0], size=params.shape)
        if mask is not None:
            z *= mask
        dg += z * jtvp(cache, params, bands, L, jvp(cache, params, bands, L, z, precision, nmax, slab), precision, nmax, slab)
    dg = np.abs(dg) / max(int(probes), 1)
    return np.maximum(dg, 1e-6 * dg.max()) if dg.max() > 0 else dg


def lsqr(Av, Atu, r, damp=0.0, iterations=40, atol=1e-6):
    """LSQR (Paige & Saunders 1982) for min |A x + r|^2 + damp^2 |x|^2 from the products A v and
    A^T u, the recurrences in FP64 (the loop of lsqr_step!, gauss_newton.jl:326-357). Returns
    (x, iterations taken, |A^T r_k| / |A^T r_0|)."""
    u = -np.asarray(r, dtype=np.float64)
    beta = float(np.linalg.norm(u))
    v0 = Atu(np.zeros_like(u)) if beta == 0 else None
    if beta == 0:
        return np.zeros_like(v0), 0, 0.0
    u /= beta
    v = np.asarray(Atu(u), dtype=np.float64)
    alpha = float(np.linalg.norm(v))
    x = np.zeros_like(v)
    if alpha == 0:
        return x, 0, 0.0
    v /= alpha
    w = v.copy()
    phibar, rhobar = beta, alpha
    norm0 = alpha * beta
    rel, k = 1.0, 0
    for it in range(1, int(iterations) + 1):
        k = it
        u = np.asarray(Av(v), dtype=np.float64) - alpha * u
        beta = float(np.linalg.norm(u))
        if beta > 0:
            u /= beta
        v = np.asarray(Atu(u), dtype=np.float64) - beta * v
        alpha = float(np.linalg.norm(v))
        if alpha > 0:
            v /= alpha
        rhohat = np.hypot(rhobar, damp)            # the damping's rotation
        chat = rhobar / rhohat
        phibar = chat * phibar
        rho = np.hypot(rhohat, beta)               # the bidiagonal's rotation
        c, s = rhohat / rho, beta / rho
        theta = s * alpha
        rhobar = -c * alpha
        phi = c * phibar
        phibar = s * phibar
        x += (phi / rho) * w
        w = v - (theta / rho) * w
        rel = abs(phibar * alpha * c) / norm0      # |A^T r_k| / |A^T r_0|
        if rel <= atol or beta == 0 or alpha == 0:
            break
    return x, k, rel


def lsqr_step(cache, params, bands, L, r, scale, damp=0.0, iterations=40, atol=1e-6, precision=KS_MIXED, nmax=-1, slab=0.0):
    """The damped least-squares step min |J S x + r|^2 + damp^2 |x|^2 on the column-scaled Jacobian
    (lsqr_step!, gauss_newton.jl:326-357): J v by `jvp`, J^T u by `jtvp`, one of each per iteration.
    `scale` is S, parameter-shaped (a zero fixes a parameter); the step is S x. Returns
    (x (21, nsplat), iterations, relative normal-equation residual)."""
    S = np.asarray(scale, dtype=np.float64)
    Av = lambda v: jvp(cache, params, bands, L, S * v.reshape(S.shape), precision, nmax, slab)
    Atu = lambda u: (S * jtvp(cache, params, bands, L, u, precision, nmax, slab)).ravel()
    x, k, rel = lsqr(Av, Atu, r, damp=damp, iterations=iterations, atol=atol)
    return x.reshape(S.shape), k, rel


def polish_timeresolved(cache, params, bands, L, iterations=5, solve_iterations=40, lam=1e-2, probes=8, probe_every=4, free=None, rng=None,
                        precision=KS_MIXED, nmax=-1, slab=0.0, callback=None):
    """Levenberg-Marquardt steps on the splat parameters against the scans (polish_timeresolved!,
    gauss_newton.jl:361-412): each step solves (J^T J + lam D) p = -J^T r by LSQR on J D^(-1/2) with
    damp = sqrt(lam), D the Hutchinson diagonal (refreshed every `probe_every` steps; |J^T r| with
    probes = 0); lam / 3 when the gain ratio exceeds 0.75, x 2 below 0.25, x 10 and the step rejected
    when chi^2 rises. Returns (params, chi^2 history)."""
    rng = np.random.default_rng(0) if rng is None else rng
    params = np.array(params, dtype=np.float64)
    mask = np.ones_like(params) if free is None else np.asarray(free, dtype=np.float64)
    r, chi = residuals(cache, params, bands, L, precision, nmax, slab)
    history = [chi]
    damping = float(lam)
    dscale = None
    for it in range(1, int(iterations) + 1):
        g = jtvp(cache, params, bands, L, r, precision, nmax, slab) * mask
        if probes > 0:
            if it == 1 or (it - 1) % max(int(probe_every), 1) == 0:
                dscale = normal_diagonal(cache, params, bands, L, probes, rng, mask, precision, nmax, slab)
        else:
            dscale = np.maximum(np.abs(g), np.finfo(np.float32).eps)
        S = mask / np.sqrt(dscale)
        x, ksolve, rel = lsqr_step(cache, params, bands, L, r, S, damp=np.sqrt(damping), iterations=solve_iterations, precision=precision,
                                   nmax=nmax, slab=slab)
        p = S * x
        Jp = jvp(cache, params, bands, L, p, precision, nmax, slab)
        predicted = chi - float((r + Jp) @ (r + Jp))
        trial = params + p
        rt, chit = residuals(cache, trial, bands, L, precision, nmax, slab)
        gain = (chi - chit) / max(predicted, np.finfo(float).eps)
        if chit < chi:
            params, r, chi = trial, rt, chit
            damping = max(damping / 3, 1e-8) if gain > 0.75 else (damping * 2 if gain < 0.25 else damping)
        else:
            damping *= 10
        history.append(chi)
        if callback is not None:
            callback(it, params, chi, damping, dict(gain=gain, predicted=predicted, solve_iterations=ksolve, solve_residual=rel))
    return params, history


def dual_valgrad(cache, params, times, nus, L, data, sigma, mask=None, precision=KS_MIXED, nmax=-1, slab=0.0):
    """chi^2 and its gradient at host parameters through one ks_chi2_gradient call (fit!'s
    _dual_valgrad, Fit.jl:422-434, with the image-domain seed on the device in place of the host
    _frame_seed! round trip). Returns (chi2, grad (21, nsplat))."""
    chi, g = chi2_gradient(cache, PolarizedSplats(params), times, nus, L, data, sigma, mask=mask, nmax=nmax, slab=slab, precision=precision)
    return chi, np.asarray(g)


class GraphValgrad:
    """dual_valgrad with the mixed evaluation captured once as a CUDA graph (capture_chi2_gradient):
    each call writes the parameters into the model's device buffer, replays the graph, and reads
    chi^2 and the gradient back. That is one host-to-device copy of the parameters, one replay and
    one device-to-host copy of the gradient per evaluation, with no validation, table staging or
    launch setup on the host. Same values as dual_valgrad(..., precision=KS_MIXED) bit for bit. The
    data, sigma and mask are copied to the device once."""

    def __init__(self, cache, params, times, nus, L, data, sigma, mask=None, nmax=-1, slab=0.0):
        import torch
        params = np.asarray(params, dtype=np.float64)
        self.nsplat = params.shape[1]
        self.model = PolarizedSplats(torch.tensor(params, device="cuda"))
        self.data = torch.as_tensor(np.asarray(data, dtype=np.float64), device="cuda")
        self.sigma = sigma if np.isscalar(sigma) else torch.as_tensor(np.asarray(sigma, dtype=np.float64), device="cuda")
        self.mask = None if mask is None else torch.as_tensor(np.ascontiguousarray(mask, dtype=np.uint8), device="cuda")
        self.graph = capture_chi2_gradient(cache, self.model, times, nus, L, self.data, self.sigma, mask=self.mask, nmax=nmax, slab=slab)

    def __call__(self, params):
        import torch
        # the model's device buffer is the column-major copy: (nsplat, 21) row-major
        self.model.sets()[0].params.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(params, dtype=np.float64).T)))
        chi2, dp = self.graph.replay()
        return float(chi2.item()), dp.cpu().numpy().reshape(self.nsplat, 21).T.copy()

    def close(self):
        self.graph.close()


class Adam:
    """The Adam step of the fit loop (Kingma & Ba 2015), on the host as in the reference's
    _fit_loop!: m, v moment estimates with bias correction."""

    def __init__(self, shape, lr=1e-2, beta1=0.9, beta2=0.999, eps=1e-8):
        self.lr, self.b1, self.b2, self.eps = float(lr), float(beta1), float(beta2), float(eps)
        self.m = np.zeros(shape)
        self.v = np.zeros(shape)
        self.t = 0

    def step(self, params, grad):
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * grad
        self.v = self.b2 * self.v + (1 - self.b2) * grad * grad
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return params - self.lr * mh / (np.sqrt(vh) + self.eps)


def fit(valgrad, params, iterations=100, lr=1e-2, scale=None, callback=None):
    """A minimal fit loop: `iterations` Adam steps on `valgrad(params) -> (chi2, grad)` (the
    device value-and-gradient, e.g. `dual_valgrad` bound to a cache and data), optionally in the
    per-parameter units `scale` (the optimiser works on params / scale; a zero scale holds that
    parameter). Returns (params, history) with the chi^2 at the start of every iteration (fit!'s
    `history`)."""
    p0 = np.array(params, dtype=np.float64)
    sc = np.ones_like(p0) if scale is None else np.broadcast_to(np.asarray(scale, dtype=np.float64), p0.shape)
    free = sc != 0
    unit = np.where(free, sc, 1.0)
    z = np.where(free, p0 / unit, 0.0)
    opt = Adam(p0.shape, lr=lr)
    history = []
    p = p0
    for it in range(int(iterations)):
        chi, g = valgrad(p)
        history.append(chi)
        z = opt.step(z, np.where(free, g * sc, 0.0))
        p = np.where(free, z * unit, p0)
        if callback is not None:
            callback(it, p, chi)
    return p, history
