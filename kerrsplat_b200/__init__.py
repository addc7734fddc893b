"""kerrsplat_b200 -- the B200 render hot path of KerrSplat behind the reference's interface.

Python mirror of the reference's Geodesics/Splats API for this path (names follow the Julia
functions without the `!`):

    cam = Camera((-15, 15), (-15, 15), 128)             # camera.jl:19-46
    cache = GeodesicCache(cam, 512)                      # cache.jl:106-125 (fused mode: no samples)
    regenerate(cache, 0.94, np.deg2rad(17), marcher=Fused(64))   # cache.jl:153-180
    img = thin_image(cache, params14, t_obs)             # Splats.jl:137-147
    stokes = polarized_image(cache, PolarizedSplats(p21), t_obs, 230e9, L)   # polarized.jl:174-179
    cube = polarized_cube(cache, PolarizedSplats(p21), times, nus, L)         # polarized.jl:187-198

Every call runs on the GPU through libkerrsplat_b200.so (ctypes, include/kerrsplat_b200.h); there
is no CPU fallback. Parameter matrices are (NROWS, nsplat) like the reference's column-major
`p[row, i]`; numpy arrays, CPU tensors and CUDA tensors are accepted.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import KS_FP64, KS_MIXED, KS_MIXED_GEO64, KsError

__all__ = [
    "Camera", "GeodesicCache", "Fused", "Recurrence", "regenerate", "thin_image", "thin_image_sorted",
    "polarized_image", "polarized_cube", "render", "capture_render", "RenderGraph", "capture_chi2_gradient", "Chi2GradientGraph", "KnotSplats", "adjoint", "chi2_gradient", "sweep_passes", "sample_adjoint", "jvp", "normal_matrix", "spacetime_derivatives", "vis_chi2_gradient", "autotune", "thin_image_noalloc", "RIAFModel", "riaf_image", "visibilities", "vis_seed", "frame_chi2_seed", "PolarizedSplats", "PowerLawSplats", "KappaSplats",
    "CompositeModel", "to_screen", "unsort", "gravitational_radius", "flux_density", "pixel_solid_angle",
    "KS_FP64", "KS_MIXED", "KS_MIXED_GEO64", "KsError", "NU0",
]

# constants.jl:3-12 and coefficients.jl:299
GNEWT, MSUN, CL, JY = 6.6742e-8, 1.989e33, 2.99792458e10, 1e-23
NU0 = 1e11


def gravitational_radius(M_solar):
    """L = GM/c^2 in cm (transport.jl:58)."""
    return GNEWT * M_solar * MSUN / (CL * CL)


def pixel_solid_angle(dalpha, L, D):
    """Solid angle of a square pixel of side `dalpha` M (transport.jl:125)."""
    return (dalpha * L / D) ** 2


def flux_density(img, dalpha, L, D):
    """Flux density per pixel in Jy (polarized.jl:201)."""
    return np.asarray(img) * (pixel_solid_angle(dalpha, L, D) / JY)


class Camera:
    """Bardeen screen (camera.jl:19-46): `Camera((amin, amax), (bmin, bmax), res)` builds Krang's
    endpoint-inclusive grid in column-major order (alpha fastest); `Camera(alphas, betas)` is an
    arbitrary point set of shape (npix, 1)."""

    def __init__(self, a, b, res=None):
        if res is None:
            self.alpha = np.ascontiguousarray(a, dtype=np.float64).ravel()
            self.beta = np.ascontiguousarray(b, dtype=np.float64).ravel()
            if self.alpha.size != self.beta.size:
                raise ValueError("camera pixel vectors do not match the screen size")
            self.size = (self.alpha.size, 1)
            return
        na, nb = (res, res) if np.isscalar(res) else res
        av = self.grid_axis(float(a[0]), float(a[1]), int(na))
        bv = self.grid_axis(float(b[0]), float(b[1]), int(nb))
        self.alpha = np.tile(av, nb)
        self.beta = np.repeat(bv, na)
        self.size = (int(na), int(nb))

    @staticmethod
    def grid_axis(lo, hi, n):
        """camera.jl:123-124, evaluated the same way so that pixels agree bit for bit."""
        if n == 1:
            return np.array([lo])
        return np.array([lo + (hi - lo) * (float(i) - 1.0) / (n - 1) for i in range(1, n + 1)])

    @property
    def npix(self):
        return self.alpha.size


class Fused:
    """Fused(M): the march runs inside the consumer, re-anchored every M samples (cache.jl:57-61)."""

    def __init__(self, M=64):
        self.M = int(M)


class Recurrence(Fused):
    """Recurrence(M): the same march; stored samples are produced on demand by `cache.samples()`."""


def _ptr(x):
    """Device or host address of a contiguous float64 buffer (numpy array or torch tensor)."""
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data)


def _as_f64(x):
    if hasattr(x, "data_ptr"):
        import torch
        return x.to(torch.float64).contiguous()
    return np.ascontiguousarray(x, dtype=np.float64)


def _colmajor(p, nrows):
    """(nrows, nsplat) parameter matrix -> contiguous buffer in column-major order.

    For a CUDA tensor the transposed copy runs on torch's current stream; the library reads it on
    its own non-blocking stream, so the copy is waited for here before the buffer is handed over."""
    if hasattr(p, "data_ptr"):
        import torch
        if p.dim() != 2 or p.shape[0] != nrows:
            raise ValueError(f"parameter matrix must be {nrows} x nsplat, got {tuple(p.shape)}")
        buf = p.to(torch.float64).t().contiguous()
        if buf.is_cuda:
            torch.cuda.current_stream(buf.device).synchronize()
        return buf, int(p.shape[1])
    p = np.asarray(p, dtype=np.float64)
    if p.ndim != 2 or p.shape[0] != nrows:
        raise ValueError(f"parameter matrix must be {nrows} x nsplat, got {p.shape}")
    return np.ascontiguousarray(p.T), int(p.shape[1])


class GeodesicCache:
    """Device-resident geodesic data for one camera and `nsamples` samples per ray (cache.jl:85-125):
    the per-ray FP64 constants in root-case-sorted order, the permutation and case ranges, the FP64
    anchor table, and the anchor residuals of the last FP64 march."""

    def __init__(self, camera, nsamples, device=0):
        if nsamples < 1:
            raise ValueError("need at least one sample per ray")
        self._lib = _lib.load()
        ctx = ctypes.c_void_p()
        st = self._lib.ks_context_create(int(device), 0, ctypes.byref(ctx))
        if st != _lib.KS_OK:
            raise KsError(st, f"cannot create a context on CUDA device {device} (status {st})")
        self._ctx = ctx
        self.nsamples = int(nsamples)
        self.camera = None
        self.spin = float("nan")
        self.theta_o = float("nan")
        self.generation = 0
        self.marcher = None
        self.set_camera(camera)

    def _check(self, status):
        _lib.check(status, self._ctx)

    def set_camera(self, camera):
        self.camera = camera
        na, nb = camera.size
        self._check(self._lib.ks_camera_set(self._ctx, _ptr(camera.alpha), _ptr(camera.beta), camera.npix, na, nb))
        self.generation = 0

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.ks_context_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def npix(self):
        return self.camera.npix

    @property
    def size(self):
        return self.camera.size

    @property
    def nsamples_per_ray(self):
        """Sample count of every ray in sorted order (all cache.nsamples unless regenerated uneven)."""
        out = np.empty(self.npix, dtype=np.int32)
        self._check(self._lib.ks_get_nsamples(self._ctx, _ptr(out)))
        return out

    @property
    def perm(self):
        """perm[j] = screen index (0-based) of sorted slot j."""
        out = np.empty(self.npix, dtype=np.int64)
        self._check(self._lib.ks_get_perm(self._ctx, _ptr(out)))
        return out

    @property
    def ranges(self):
        """Half-open sorted-slot ranges of the three root cases (4, 2, 0 real roots)."""
        r = np.empty(6, dtype=np.int64)
        self._check(self._lib.ks_get_ranges(self._ctx, _ptr(r)))
        return {"case2": range(r[0], r[1]), "case3": range(r[2], r[3]), "case4": range(r[4], r[5])}

    def residuals(self):
        rt = np.empty(self.npix)
        rp = np.empty(self.npix)
        self._check(self._lib.ks_get_residuals(self._ctx, _ptr(rt), _ptr(rp)))
        return rt, rp

    def ray_constants(self):
        """npix x 24 FP64 per-ray constants in sorted order (see ks_get_ray_constants)."""
        out = np.empty((self.npix, 24))
        self._check(self._lib.ks_get_ray_constants(self._ctx, _ptr(out)))
        return out

    def samples(self):
        """Recurrence(M) stored mode (quadrature.jl:336-348): dict of (N, npix) arrays t, r, theta,
        phi, flags in sorted order (the reference's (npix, N) column-major matrices)."""
        N, n = self.nsamples, self.npix
        t, r, th, ph = (np.empty((N, n)) for _ in range(4))
        fl = np.empty((N, n), dtype=np.uint8)
        self._check(self._lib.ks_march_samples(self._ctx, _ptr(t), _ptr(r), _ptr(th), _ptr(ph), _ptr(fl)))
        return {"t": t, "r": r, "theta": th, "phi": ph, "flags": fl}

    def kernel_stats(self, reset=False):
        ms = ctypes.c_double()
        kl = ctypes.c_longlong()
        al = ctypes.c_longlong()
        self._check(self._lib.ks_kernel_stats(self._ctx, ctypes.byref(ms), ctypes.byref(kl), ctypes.byref(al), int(reset)))
        return ms.value, kl.value, al.value

    def set_stage_test(self, on):
        """Test hook: while on, mixed calls fail with a timeout of the table-staging wait (no fault)."""
        self._check(self._lib.ks_set_stage_test(self._ctx, int(bool(on))))

    def set_tensor_path(self, path):
        """Kernel of the 3xTF32 GEMMs: "tcgen05" (UMMA, the default) or "mma.sync" (the fallback)."""
        code = {"tcgen05": 0, "mma.sync": 1}[path]
        self._check(self._lib.ks_set_tensor_path(self._ctx, code))

    def gemm_stats(self, reset=False):
        """(ms, launches, flops) of the 3xTF32 GEMMs since the last reset (CUDA events, device time)."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        fl = ctypes.c_double()
        self._check(self._lib.ks_gemm_stats(self._ctx, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(fl), int(reset)))
        return ms.value, n.value, fl.value

    def consume_stats(self, reset=False):
        """(ms, launches) of k_consume alone in the mixed renders since the last reset."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._check(self._lib.ks_consume_stats(self._ctx, ctypes.byref(ms), ctypes.byref(n), int(reset)))
        return ms.value, n.value

    def count_events(self, on=True):
        self._check(self._lib.ks_set_event_counting(self._ctx, int(on)))

    def event_counts(self):
        """Work events of the last counted ks_render: samples (per combination), valid samples,
        splat tests, weights evaluated, coefficient evaluations, frames, transfer steps."""
        out = np.zeros(7, dtype=np.uint64)
        self._check(self._lib.ks_event_counts(self._ctx, _ptr(out)))
        keys = ("samples", "valid_samples", "splat_tests", "weights", "coefficients", "frames", "steps")
        return dict(zip(keys, (int(v) for v in out)))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self._lib.ks_context_stream(self._ctx, ctypes.byref(s)))
        return s.value


def regenerate(cache, a, theta_o, camera=None, marcher=None, uneven=None):
    """regenerate!(cache, a, theta_o[, camera]; marcher) (cache.jl:153-180, 248-255). With
    `uneven = (samples_per_mino, nmin)` every ray gets its own sample count
    N_j = clamp(64 ceil(samples_per_mino tau_total_j / 64), nmin, cache.nsamples)."""
    if camera is not None:
        if camera.npix != cache.npix:
            raise ValueError(f"camera has {camera.npix} pixels, cache was built for {cache.npix}")
        cache.set_camera(camera)
    marcher = marcher or Fused(64)
    if uneven is None:
        cache._check(cache._lib.ks_regenerate(cache._ctx, float(a), float(theta_o), cache.nsamples, marcher.M))
    else:
        density, nmin = uneven
        cache._check(cache._lib.ks_regenerate_uneven(cache._ctx, float(a), float(theta_o), float(density), int(nmin), cache.nsamples,
                                                     marcher.M))
    cache.spin, cache.theta_o, cache.marcher = float(a), float(theta_o), marcher
    cache.generation += 1
    return cache


def _precision(p):
    if p in (KS_FP64, "fp64", "float64"):
        return KS_FP64
    if p in (KS_MIXED, "mixed", "fp32"):
        return KS_MIXED
    if p in (KS_MIXED_GEO64, "mixed_geo64"):
        return KS_MIXED_GEO64
    raise ValueError(f"unknown precision {p!r}")


def _out_like(x, shape):
    if hasattr(x, "data_ptr") and x.is_cuda:
        import torch
        return torch.empty(shape, dtype=torch.float64, device=x.device)
    return np.empty(shape)


def thin_image_sorted(cache, params, t_obs, precision=KS_FP64, out=None):
    """thin_image!(out, cache, params, t_obs) (Splats.jl:137-140): sorted-order Stokes I."""
    buf, ns = _colmajor(params, 14)
    out = _out_like(buf, cache.npix) if out is None else out
    cache._check(cache._lib.ks_thin_image(cache._ctx, _ptr(buf), ns, float(t_obs), _precision(precision), _ptr(out), _lib.KS_ORDER_SORTED))
    return out


def thin_image(cache, params, t_obs, precision=KS_FP64):
    """Screen-shaped optically-thin image (Splats.jl:143-147): shape (nalpha, nbeta) in the
    reference's column-major sense, i.e. img[i, j] is pixel i + j * nalpha."""
    buf, ns = _colmajor(params, 14)
    out = _out_like(buf, cache.npix)
    cache._check(cache._lib.ks_thin_image(cache._ctx, _ptr(buf), ns, float(t_obs), _precision(precision), _ptr(out), _lib.KS_ORDER_SCREEN))
    na, nb = cache.size
    return out.reshape(nb, na).T if isinstance(out, np.ndarray) else out.reshape(nb, na).t()


def thin_image_noalloc(cache, params, t_obs, out, precision=KS_FP64, order="sorted"):
    """ks_thin_image_noalloc: the thin image with no device allocation inside the call, for callers
    whose device memory is owned by their own allocator. `params` is a (14, nsplat) CUDA tensor, as
    for thin_image_sorted, and `out` an (npix,) float64 CUDA tensor; at most KS_NOALLOC_MAX_SPLATS
    splats. The library runs on its own stream, so pending work on torch's current stream (the
    writers of `params` and `out`) is waited for before the call."""
    buf, ns = _colmajor(params, 14)
    if hasattr(out, "is_cuda") and out.is_cuda:
        import torch
        torch.cuda.current_stream(out.device).synchronize()
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_thin_image_noalloc(cache._ctx, _ptr(buf), ns, float(t_obs), _precision(precision), _ptr(out), o))
    return out


class _Model:
    kind = None

    def sets(self):
        return [self]


class PolarizedSplats(_Model):
    """Thermal splats, 21 rows (polarized.jl:17-19, 41-49)."""
    kind = _lib.KS_THERMAL21

    def __init__(self, params):
        self.params, self.nsplat = _colmajor(params, 21)


class PowerLawSplats(_Model):
    """Power-law splats, 22 rows, common gamma_max (populations.jl:34-41)."""
    kind = _lib.KS_POWERLAW22

    def __init__(self, params, gamma_max=1e5):
        self.params, self.nsplat = _colmajor(params, 22)
        self.gamma_max = float(gamma_max)


def kappa_hypergeometric(kappa, w):
    """2F1(kappa - 1/3, kappa + 1, kappa + 2/3, -kappa w), host side (kappa.jl:97-100)."""
    import mpmath
    return float(mpmath.hyp2f1(kappa - 1.0 / 3, kappa + 1.0, kappa + 2.0 / 3, -kappa * w))


class KappaSplats(_Model):
    """kappa splats, 22 rows; the hypergeometric factors are computed on the host
    (populations.jl:50-60)."""
    kind = _lib.KS_KAPPA22

    def __init__(self, params, hyp=None):
        self.params, self.nsplat = _colmajor(params, 22)
        if hyp is None:
            hp = np.asarray(params if not hasattr(params, "cpu") else params.cpu().numpy(), dtype=np.float64)
            hyp = [kappa_hypergeometric(hp[13, i], np.exp(hp[14, i])) for i in range(hp.shape[1])]
        self.hyp = np.ascontiguousarray(hyp, dtype=np.float64)


class KnotSplats(_Model):
    """Thermal splats whose centres follow trajectory knots (trajectories.jl:80-129): `params` 21 rows
    (rows 1-3 and the pattern rate are not used), `knots` (3, nknots, nsplat) quasi-Cartesian
    Kerr-Schild centres at the increasing coordinate `times` (nknots); the centre at a sample's
    emission time is interpolated linearly and clamped to the end knots."""
    kind = _lib.KS_KNOT21

    def __init__(self, params, knots, times):
        self.params, self.nsplat = _colmajor(params, 21)
        k = np.asarray(knots, dtype=np.float64)
        t = np.ascontiguousarray(times, dtype=np.float64).ravel()
        if k.ndim != 3 or k.shape[0] != 3 or k.shape[1] != t.size or k.shape[2] != self.nsplat:
            raise ValueError(f"knots must be (3, {t.size}, {self.nsplat}), got {k.shape}")
        if t.size > 1 and not np.all(np.diff(t) > 0):
            raise ValueError("knot times must increase")
        self.knots = np.ascontiguousarray(k.ravel(order="F"))   # x fastest, then knot, then splat
        self.knot_times = t
        self.nknots = int(t.size)


class CompositeModel(_Model):
    """Union of models (transport.jl:348-358): the elements of `a` followed by those of `b`."""

    def __init__(self, *models):
        self.models = models

    def sets(self):
        out = []
        for m in self.models:
            out.extend(m.sets())
        return out


def _set_array(model):
    sets = model.sets()
    arr = (_lib.SplatSetC * max(1, len(sets)))()
    keep = []
    for i, m in enumerate(sets):
        arr[i].kind = m.kind
        arr[i].nsplat = m.nsplat
        arr[i].params = _ptr(m.params).value
        hyp = getattr(m, "hyp", None)
        arr[i].hyp = _ptr(hyp).value if hyp is not None else None
        kn = getattr(m, "knots", None)
        arr[i].knots = _ptr(kn).value if kn is not None else None
        arr[i].knot_times = _ptr(m.knot_times).value if kn is not None else None
        arr[i].nknots = getattr(m, "nknots", 0)
        arr[i].gamma_max = getattr(m, "gamma_max", 1e5)
        keep.append(m)
    return arr, len(sets), keep


def render(cache, model, times, nus, L, nmax=-1, slab=0.0, precision=KS_FP64, order="screen", out=None):
    """Stokes (I, Q, U, V) in cgs for every (frame, frequency): array (nfreq, nframes, npix, 4) in
    screen (camera) or sorted order. One GPU call (ks_render)."""
    times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
    nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
    nt, nf = int(times.shape[0]), int(nus.shape[0])
    arr, nsets, _keep = _set_array(model)
    if out is None:
        out = _out_like(model.sets()[0].params if nsets else times, (nf, nt, cache.npix, 4))
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_render(cache._ctx, arr, nsets, _ptr(times), nt, _ptr(nus), nf, float(L), _precision(precision),
                                      int(nmax), float(slab), _ptr(out), o))
    return out


class RenderGraph:
    """A mixed render captured as a CUDA graph (ks_render_graph_capture): replay() re-renders into
    `out` from the current values of the model's device parameter buffers, model.sets()[i].params
    (column-major copies the model made of the matrices it was given; update those in place, e.g.
    model.sets()[0].params[:, 12] += 0.1 for the log density of a thermal set). Frames, frequencies,
    L, the splat counts and the knots are fixed at capture."""

    def __init__(self, cache, model, times, nus, L, out, nmax, slab, order):
        self.cache, self.model, self.out = cache, model, out
        times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
        nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
        arr, nsets, self._keep = _set_array(model)
        o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
        cache._check(cache._lib.ks_render_graph_capture(cache._ctx, arr, nsets, _ptr(times), int(times.shape[0]), _ptr(nus),
                                                        int(nus.shape[0]), float(L), int(nmax), float(slab), _ptr(out), o))

    def replay(self, wait=True):
        self.cache._check(self.cache._lib.ks_graph_launch(self.cache._ctx, int(bool(wait))))
        return self.out

    def close(self):
        self.cache._check(self.cache._lib.ks_graph_destroy(self.cache._ctx))


def capture_render(cache, model, times, nus, L, out=None, nmax=-1, slab=0.0, order="screen"):
    """Capture one mixed render of a device-resident model (torch CUDA tensors) as a CUDA graph; the
    returned RenderGraph replays it with no host work (the forward pass of a fit iteration)."""
    nt = len(np.atleast_1d(times)) if not hasattr(times, "data_ptr") else int(times.shape[0])
    nf = len(np.atleast_1d(nus)) if not hasattr(nus, "data_ptr") else int(nus.shape[0])
    if out is None:
        out = _out_like(model.sets()[0].params, (nf, nt, cache.npix, 4))
    return RenderGraph(cache, model, times, nus, L, out, nmax, slab, order)


class Chi2GradientGraph:
    """One mixed chi^2 + gradient evaluation captured as a CUDA graph (ks_chi2_gradient_graph_capture):
    replay() recomputes chi2 (a one-element device tensor) and dparams (a device tensor laid out as
    chi2_gradient's dparams) from the current values of the model's device parameter buffers,
    model.sets()[i].params, and of the data. The fit loop's evaluation with no host work: update the
    parameters in place on the device, replay, read chi2 and dparams on the device."""

    def __init__(self, cache, model, times, nus, L, data, sigma, mask, chi2, dparams, nmax, slab, accumulate):
        self.cache, self.model, self.chi2, self.dparams = cache, model, chi2, dparams
        times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
        nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
        self._keep = [data, sigma, mask]
        arr, nsets, self._keep_sets = _set_array(model)
        sg, ss = (None, float(sigma)) if np.isscalar(sigma) else (sigma, 0.0)
        cache._check(cache._lib.ks_chi2_gradient_graph_capture(
            cache._ctx, arr, nsets, _ptr(times), int(times.shape[0]), _ptr(nus), int(nus.shape[0]), float(L), int(nmax), float(slab),
            _ptr(data), _ptr(sg) if sg is not None else None, ss, _ptr(mask) if mask is not None else None, _ptr(chi2), _ptr(dparams),
            int(bool(accumulate))))

    def replay(self, wait=True):
        self.cache._check(self.cache._lib.ks_chi2_gradient_graph_launch(self.cache._ctx, int(bool(wait))))
        return self.chi2, self.dparams

    def close(self):
        self.cache._check(self.cache._lib.ks_graph_destroy(self.cache._ctx))


def capture_chi2_gradient(cache, model, times, nus, L, data, sigma, mask=None, nmax=-1, slab=0.0, accumulate=False):
    """Capture one mixed chi^2 + gradient evaluation of a device-resident thermal model against
    device-resident data (torch CUDA tensors; sigma a tensor of data's shape or a scalar, mask uint8
    (nfreq, nframes, npix)). Returns a Chi2GradientGraph whose replay() fills its `chi2` (one float64)
    and `dparams` (sum of 21 x nsplat per set, float64) tensors on the device."""
    import torch
    dev = data.device
    ntot = sum(s.nsplat for s in model.sets())
    chi2 = torch.zeros(1, dtype=torch.float64, device=dev)
    dparams = torch.zeros(21 * ntot, dtype=torch.float64, device=dev)
    return Chi2GradientGraph(cache, model, times, nus, L, data, sigma, mask, chi2, dparams, nmax, slab, accumulate)


def _grad_like(model):
    """dparams of a model: one (21, nsplat) float64 array per set, concatenated column-major."""
    return [np.zeros((_lib.NROWS[s.kind], s.nsplat)) for s in model.sets()]


def _grad_buffer(model, dparams):
    if dparams is None:
        return None, np.zeros(sum(_lib.NROWS[s.kind] * s.nsplat for s in model.sets()))
    if hasattr(dparams, "data_ptr"):
        return dparams, dparams
    d = np.asarray(dparams)
    if d.dtype != np.float64 or not (d.ndim == 1 or (d.ndim == 2 and d.flags.f_contiguous)):
        raise ValueError("dparams must be a float64 array laid out like the parameters (flat, or 21 x nsplat column-major)")
    return dparams, d


def _split_grad(model, flat):
    out, q = [], 0
    for s in model.sets():
        nr = _lib.NROWS[s.kind]
        out.append(np.asarray(flat[q:q + nr * s.nsplat]).reshape(s.nsplat, nr).T.copy())
        q += nr * s.nsplat
    return out[0] if len(out) == 1 else out


def adjoint(cache, model, times, nus, L, dstokes, nmax=-1, slab=0.0, precision=KS_FP64, order="screen", dparams=None):
    """The gradient of sum(dstokes * Stokes) with respect to every splat parameter (the dual sweep,
    dual_gradient.jl:190-249): `dstokes` has the shape of `render`'s output, (nfreq, nframes, npix, 4).
    Returns (21, nsplat) per set; with `dparams` given (float64, the parameters' layout) the gradient
    is added to it in place (the reference's `dparams .+= ...`). Thermal polarized splats only."""
    times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
    nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
    nt, nf = int(times.shape[0]), int(nus.shape[0])
    ds = _as_f64(dstokes)
    if tuple(ds.shape) != (nf, nt, cache.npix, 4):
        raise ValueError(f"dstokes must have shape {(nf, nt, cache.npix, 4)}, got {tuple(ds.shape)}")
    arr, nsets, _keep = _set_array(model)
    user, buf = _grad_buffer(model, dparams)
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_adjoint(cache._ctx, arr, nsets, _ptr(times), nt, _ptr(nus), nf, float(L), _precision(precision), int(nmax),
                                       float(slab), _ptr(ds), o, _ptr(buf), 1 if user is not None else 0))
    return user if user is not None else _split_grad(model, buf)


def chi2_gradient(cache, model, times, nus, L, data, sigma, mask=None, nmax=-1, slab=0.0, precision=KS_FP64, dparams=None,
                  return_image=False):
    """chi2_gradient! (Fit.jl:502-534) for image-domain data: chi^2 = sum ((image - data)/sigma)^2 over
    unmasked pixels, Stokes, frames and frequencies, and its gradient with respect to every splat
    parameter, in one forward and one reverse pass on the GPU. `data` (and `sigma` unless it is a
    scalar) have the shape of `render`'s screen-order output; `mask` is (nfreq, nframes, npix) bools.
    Returns (chi2, grad) -- grad as `adjoint` returns it -- and the model image with `return_image`."""
    times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
    nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
    nt, nf = int(times.shape[0]), int(nus.shape[0])
    shape = (nf, nt, cache.npix, 4)
    d = _as_f64(data)
    if tuple(d.shape) != shape:
        raise ValueError(f"data must have shape {shape}, got {tuple(d.shape)}")
    if np.isscalar(sigma):
        sg, ss = None, float(sigma)
        if not (np.isfinite(ss) and ss > 0):
            raise ValueError("sigma must be positive")
    else:
        sg, ss = _as_f64(sigma), 0.0
        if tuple(sg.shape) != shape:
            raise ValueError(f"sigma must have shape {shape}, got {tuple(sg.shape)}")
    mk = None
    if mask is not None:
        mk = np.ascontiguousarray(mask, dtype=np.uint8) if not hasattr(mask, "data_ptr") else mask
        if tuple(mk.shape) != shape[:3]:
            raise ValueError(f"mask must have shape {shape[:3]}")
    arr, nsets, _keep = _set_array(model)
    user, buf = _grad_buffer(model, dparams)
    chi2 = ctypes.c_double(0.0)
    img = _out_like(d, shape) if return_image else None
    cache._check(cache._lib.ks_chi2_gradient(cache._ctx, arr, nsets, _ptr(times), nt, _ptr(nus), nf, float(L), _precision(precision),
                                             int(nmax), float(slab), _ptr(d), _ptr(sg) if sg is not None else None, ss,
                                             _ptr(mk) if mk is not None else None, ctypes.addressof(chi2), _ptr(buf),
                                             1 if user is not None else 0, _ptr(img) if img is not None else None))
    g = user if user is not None else _split_grad(model, buf)
    return (chi2.value, g, img) if return_image else (chi2.value, g)


def jvp(cache, model, times, nus, L, dirs, nmax=-1, slab=0.0, precision=KS_FP64, order="screen", return_image=False):
    """J v of the image (jvp!, gauss_newton.jl:91-118) along each direction in `dirs`: an array of
    (ndir, 21, nsplat) (or (21, nsplat) for one direction; several sets: (ndir, nparams) flat, each
    direction laid out like `adjoint`'s dparams). Returns (ndir, nfreq, nframes, npix, 4)."""
    times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
    nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
    nt, nf = int(times.shape[0]), int(nus.shape[0])
    nparams = sum(_lib.NROWS[s.kind] * s.nsplat for s in model.sets())
    d = np.asarray(dirs, dtype=np.float64)
    if d.ndim == 2 and d.shape[0] == 21 and len(model.sets()) == 1 and d.shape[1] == model.sets()[0].nsplat:
        d = d[None]
    if d.ndim == 3:   # (ndir, 21, nsplat) -> column-major per direction
        d = np.ascontiguousarray(np.transpose(d, (0, 2, 1))).reshape(d.shape[0], -1)
    d = np.ascontiguousarray(d.reshape(-1, nparams))
    nd = d.shape[0]
    arr, nsets, _keep = _set_array(model)
    out = np.empty((nd, nf, nt, cache.npix, 4))
    img = np.empty((nf, nt, cache.npix, 4)) if return_image else None
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_jvp(cache._ctx, arr, nsets, _ptr(times), nt, _ptr(nus), nf, float(L), _precision(precision), int(nmax),
                                   float(slab), _ptr(d), nd, _ptr(out), o, _ptr(img) if img is not None else None))
    return (out, img) if return_image else out


def spacetime_derivatives(cache, model, times, nus, L, nmax=-1, slab=0.0, precision=KS_FP64, return_image=False):
    """d(image)/d(a, theta_o, ln L) (the spacetime block of spacetime_valgrad, joint.jl:74-82): array
    (3, nfreq, nframes, npix, 4) in screen order, by three-partial FP64 duals through the ray
    constants, the anchors, the march and the transport at the cache's sample counts."""
    times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
    nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
    nt, nf = int(times.shape[0]), int(nus.shape[0])
    arr, nsets, _keep = _set_array(model)
    out = np.empty((3, nf, nt, cache.npix, 4))
    img = np.empty((nf, nt, cache.npix, 4)) if return_image else None
    cache._check(cache._lib.ks_spacetime_derivatives(cache._ctx, arr, nsets, _ptr(times), nt, _ptr(nus), nf, float(L), _precision(precision),
                                                     int(nmax), float(slab), _ptr(out),
                                                     _ptr(img) if img is not None else None))
    return (out, img) if return_image else out


def autotune(cache, model, times, nus, L, nmax=-1, slab=0.0, trials=2):
    """Pick the mixed forward pass's block size and work-unit density for this scene by timing every
    candidate on the GPU; later renders of the cache use the choice. Returns (block, units, ms)."""
    times = _as_f64(np.atleast_1d(times) if not hasattr(times, "data_ptr") else times)
    nus = _as_f64(np.atleast_1d(nus) if not hasattr(nus, "data_ptr") else nus)
    arr, nsets, _keep = _set_array(model)
    b, u, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
    cache._check(cache._lib.ks_autotune(cache._ctx, arr, nsets, _ptr(times), int(times.shape[0]), _ptr(nus), int(nus.shape[0]), float(L),
                                        int(nmax), float(slab), int(trials), ctypes.byref(b), ctypes.byref(u), ctypes.byref(ms)))
    return b.value, u.value, ms.value


def normal_matrix(cache, J, precision=KS_FP64):
    """normal_matrix(J) (gauss_newton.jl:486-494): J^T J of an (m, n) Jacobian on the GPU."""
    J = np.ascontiguousarray(J, dtype=np.float64)
    m, n = J.shape
    A = np.empty((n, n))
    cache._check(cache._lib.ks_normal_matrix(cache._ctx, _ptr(J), m, n, _precision(precision), _ptr(A)))
    return A


def sample_adjoint(cache, coeffs, Dl, w, R, method=0):
    """sample_adjoint (transport.jl:221-245) of n samples on the GPU (FP64): coeffs (n, 11) = (j, alpha,
    rho), Dl (n,), w and R (n, 4). Returns O (n, 4, 4), E (n, 4) and c-bar (n, 11). method 0 is the
    structured form (the mixed reverse pass), 1 the seven forward-mode duals (the FP64 reverse pass)."""
    coeffs = np.ascontiguousarray(coeffs, dtype=np.float64).reshape(-1, 11)
    n = coeffs.shape[0]
    Dl = np.ascontiguousarray(Dl, dtype=np.float64).reshape(n)
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(n, 4)
    R = np.ascontiguousarray(R, dtype=np.float64).reshape(n, 4)
    out = np.empty((n, 31))
    cache._check(cache._lib.ks_sample_adjoint(cache._ctx, n, _ptr(coeffs), _ptr(Dl), _ptr(w), _ptr(R), int(method), _ptr(out)))
    return out[:, :16].reshape(n, 4, 4), out[:, 16:20], out[:, 20:]


def vis_chi2_gradient(cache, model, t_obs, nu, L, u, v, vis, sigma, psize, scale, tap=None, gains=None, nmax=-1, slab=0.0,
                      precision=KS_MIXED, dparams=None, return_image=False):
    """The visibility chi^2 of one frame and its gradient (timeresolved_gradient!'s device path,
    timeresolved.jl:115-138; frame_chi2_seed!, device_visibilities.jl:97-111) in one forward and one
    reverse pass: vis (nuv, 4) complex data, sigma (nuv, 4). Returns (chi2, grad[, image])."""
    u, v = _as_f64(u), _as_f64(v)
    nuv = int(u.shape[0])
    vi = _complex_pairs(vis)
    sg = _as_f64(sigma)
    tp = _as_f64(tap) if tap is not None else None
    gg = _complex_pairs(gains) if gains is not None else None
    arr, nsets, _keep = _set_array(model)
    user, buf = _grad_buffer(model, dparams)
    chi2 = ctypes.c_double(0.0)
    img = np.empty((cache.npix, 4)) if return_image else None
    cache._check(cache._lib.ks_vis_chi2_gradient(cache._ctx, arr, nsets, float(t_obs), float(nu), float(L), _precision(precision), int(nmax),
                                                 float(slab), nuv, _ptr(u), _ptr(v), _ptr(tp) if tp is not None else None,
                                                 _ptr(gg) if gg is not None else None, _ptr(vi), _ptr(sg), float(psize), float(scale),
                                                 ctypes.addressof(chi2), _ptr(buf), 1 if user is not None else 0,
                                                 _ptr(img) if img is not None else None))
    g = user if user is not None else _split_grad(model, buf)
    return (chi2.value, g, img) if return_image else (chi2.value, g)


def sweep_passes(cache, model, L, nmax=-1, slab=0.0, precision=KS_FP64):
    """The two passes of the gradient as closures (sweep_passes, Fit.jl:451-485): `forward(t, nu)`
    returns the model image (nfreq = 1, screen order, (npix, 4) per frame) and `reverse(dstokes, t, nu)`
    returns the gradient of sum(dstokes * image). Each pass is one GPU call; the reverse pass runs its
    own forward pass, so the pair is stateless."""
    def forward(t, nu):
        return render(cache, model, np.atleast_1d(t), [nu], L, nmax=nmax, slab=slab, precision=precision)[0]

    def reverse(dstokes, t, nu):
        ds = np.asarray(dstokes, dtype=np.float64).reshape(1, len(np.atleast_1d(t)), cache.npix, 4)
        return adjoint(cache, model, np.atleast_1d(t), [nu], L, ds, nmax=nmax, slab=slab, precision=precision)

    return forward, reverse


class RIAFModel:
    """ipole's RIAF as a fluid model (the reference's test/riaf_model.jl:11-23): density and
    temperature power laws in r with a Gaussian thick-disk profile, a toroidal field of
    equipartition-like strength, Keplerian rotation outside r_isco and the plunge inside it,
    thermal synchrotron with Pandya emissivities when `pandya`."""

    def __init__(self, nth0, Te0, disk_h, pow_nth, pow_T, Ne_unit, Te_unit, eps, r_isco, rout, pandya=True):
        self.values = np.array([nth0, Te0, disk_h, pow_nth, pow_T, Ne_unit, Te_unit, eps, r_isco, rout], dtype=np.float64)
        self.pandya = bool(pandya)

    @staticmethod
    def isco_radius(a):
        """The prograde ISCO (Bardeen, Press & Teukolsky 1972; riaf_model.jl:25-29)."""
        z1 = 1 + np.cbrt(1 - a * a) * (np.cbrt(1 + a) + np.cbrt(1 - a))
        z2 = np.sqrt(3 * a * a + z1 * z1)
        return 3 + z2 - np.copysign(np.sqrt((3 - z1) * (3 + z1 + 2 * z2)), a)

    @classmethod
    def example(cls, a=0.9375, pandya=True):
        """ipole's model/riaf/example.par (riaf_example, riaf_model.jl:31-34)."""
        return cls(1.0, 1.0, 0.1, -1.1, -0.84, 3e7, 3e11, 0.1, cls.isco_radius(a), 100.0, pandya)


def riaf_image(cache, riaf, nus, L, precision=KS_FP64, order="screen"):
    """Stokes images of a RIAFModel through the polarized consumer (stokes_image,
    test/test_polarized.jl:54-61): (nfreq, npix, 4) cgs, screen order unless order="sorted"."""
    nus = np.ascontiguousarray(np.atleast_1d(nus), dtype=np.float64)
    out = np.empty((nus.size, cache.npix, 4))
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_riaf_image(cache._ctx, _ptr(riaf.values), int(riaf.pandya), _ptr(nus), nus.size, float(L),
                                          _precision(precision), _ptr(out), o))
    return out


def polarized_image(cache, model, t_obs, nu, L, nmax=-1, slab=0.0, precision=KS_FP64):
    """Screen-shaped Stokes image (polarized.jl:174-179): shape (nalpha, nbeta, 4) in cgs."""
    if not isinstance(model, _Model):
        model = PolarizedSplats(model)
    out = render(cache, model, [t_obs], [nu], L, nmax=nmax, slab=slab, precision=precision)
    na, nb = cache.size
    return np.asarray(out).reshape(nb, na, 4).transpose(1, 0, 2)


def polarized_cube(cache, model, times, nus, L, nmax=-1, slab=0.0, precision=KS_FP64):
    """Stokes movie cube (polarized.jl:187-198): shape (nalpha, nbeta, ntimes, nfreq, 4)."""
    if not isinstance(model, _Model):
        model = PolarizedSplats(model)
    out = np.asarray(render(cache, model, times, nus, L, nmax=nmax, slab=slab, precision=precision))
    nf, nt = out.shape[0], out.shape[1]
    na, nb = cache.size
    return out.reshape(nf, nt, nb, na, 4).transpose(3, 2, 1, 0, 4)


def _complex_pairs(z):
    z = np.ascontiguousarray(z, dtype=np.complex128)
    return z.view(np.float64)


def _out_array(out, shape, dtype):
    if out is None:
        return np.empty(shape, dtype=dtype)
    if out.shape != shape or out.dtype != dtype or not out.flags.c_contiguous:
        raise ValueError(f"out must be a C-contiguous {dtype.__name__} array of shape {shape}")
    return out


def visibilities(cache, image, u, v, psize, scale, tap=None, precision=KS_MIXED, order="screen", out=None):
    """Stokes visibilities V (nuv, 4) complex of an (npix, 4) image (device_visibilities.jl:61-73):
    V_k = tap_k scale sum_j I_j exp(2 pi i (u_k l_j + v_k m_j)), l toward the east (-alpha). The mixed
    path runs the separable transform as 3xTF32 tensor-core GEMMs; KS_FP64 is the direct transform.
    `out` (optional): a (nuv, 4) complex128 array to write into (pinned host memory copies faster)."""
    img = np.ascontiguousarray(image, dtype=np.float64).reshape(cache.npix, 4)
    u = np.ascontiguousarray(u, dtype=np.float64); v = np.ascontiguousarray(v, dtype=np.float64)
    tp = None if tap is None else np.ascontiguousarray(tap, dtype=np.float64)
    out = _out_array(out, (u.size, 4), np.complex128)
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_visibilities(cache._ctx, _ptr(img), o, u.size, _ptr(u), _ptr(v), None if tp is None else _ptr(tp),
                                            float(psize), float(scale), _precision(precision), _ptr(out.view(np.float64))))
    return out


def vis_seed(cache, w, u, v, psize, scale, tap=None, precision=KS_MIXED, order="screen", out=None):
    """The adjoint of `visibilities` applied to weights w (nuv, 4) complex: seed (npix, 4)
    (seed_kernel!, device_visibilities.jl:76-88). `out` (optional): an (npix, 4) float64 array."""
    wp = _complex_pairs(w)
    u = np.ascontiguousarray(u, dtype=np.float64); v = np.ascontiguousarray(v, dtype=np.float64)
    tp = None if tap is None else np.ascontiguousarray(tap, dtype=np.float64)
    out = _out_array(out, (cache.npix, 4), np.float64)
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_vis_seed(cache._ctx, _ptr(wp), u.size, _ptr(u), _ptr(v), None if tp is None else _ptr(tp), float(psize),
                                        float(scale), _precision(precision), _ptr(out), o))
    return out


def frame_chi2_seed(cache, image, u, v, vis, sigma, psize, scale, tap=None, gains=None, precision=KS_MIXED, order="screen"):
    """frame_chi2_seed! (device_visibilities.jl:97-111): chi^2 of the (gained) model visibilities
    against the data and the adjoint seed of the weighted residuals, (chi2, seed (npix, 4))."""
    img = np.ascontiguousarray(image, dtype=np.float64).reshape(cache.npix, 4)
    u = np.ascontiguousarray(u, dtype=np.float64); v = np.ascontiguousarray(v, dtype=np.float64)
    tp = None if tap is None else np.ascontiguousarray(tap, dtype=np.float64)
    gp = None if gains is None else _complex_pairs(gains)
    dp = _complex_pairs(vis)
    sg = np.ascontiguousarray(sigma, dtype=np.float64).reshape(u.size, 4)
    seed = np.empty((cache.npix, 4))
    chi2 = ctypes.c_double()
    o = _lib.KS_ORDER_SCREEN if order == "screen" else _lib.KS_ORDER_SORTED
    cache._check(cache._lib.ks_frame_chi2_seed(cache._ctx, _ptr(img), o, u.size, _ptr(u), _ptr(v), None if tp is None else _ptr(tp),
                                               None if gp is None else _ptr(gp), _ptr(dp), _ptr(sg), float(psize), float(scale),
                                               _precision(precision), ctypes.byref(chi2), _ptr(seed)))
    return chi2.value, seed


def unsort(cache, x):
    """Sorted-order rows -> screen order (cache.jl:271-286)."""
    x = np.asarray(x)
    y = np.empty_like(x)
    y[cache.perm] = x
    return y


def to_screen(cache, x):
    """unsort followed by the screen reshape (cache.jl:293-296)."""
    y = unsort(cache, x)
    na, nb = cache.size
    return y.reshape((nb, na) + y.shape[1:]).swapaxes(0, 1)
