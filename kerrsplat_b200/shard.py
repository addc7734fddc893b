"""Ray-sharded rendering and chi^2 + gradient over ranks (one process per GPU).

Every ray is independent: the image is one pixel per ray, and the dual sweep adds each ray's
contribution into the parameter gradient (dual_gradient.jl:190-249, `dparams .+= ...`). So a screen
splits into ray shards with no exchange until the end. Each rank regenerates its own shard as a
cache of its own (a `Camera` over its pixels) and runs the ordinary entry points on it. One SUM
all-reduce of [chi^2, dparams] then gives every rank the whole screen's chi^2 and gradient: 1 + 21 x
nsplat FP64 values per thermal set (86 KB at 512 splats), latency-bound over NVLink. Forward images
need only a gather.

The rays are dealt in the root-case-sorted order of the whole screen (cache.perm,
pixel_constants.jl:167-176). "strided" (the default) deals slot j to rank j mod world, so that every
rank gets a thinned copy of the screen and of each root case, and so the same share of the rays that
cross the splats. "contiguous" gives each rank a range of that order whose sample sum (sum of N_j,
uneven N included) is within one ray's count of the total / world; it balances the march but not the
transport, whose work follows the splats. On the 256 x 256 configuration-3 scene the largest
contiguous shard takes 1.31, 1.47 and 2.08 times the whole screen's time / ranks at 2, 4 and 8
ranks, the largest strided shard 1.06, 1.11 and 1.27.

The partition is deterministic: every rank computes every rank's pixels, which the gather uses."""

import numpy as np

from . import KS_MIXED, Camera, GeodesicCache, chi2_gradient, regenerate, render
from . import _lib

__all__ = ["ray_shards", "RayShard", "chi2_gradient_shard", "chi2_gradient_sharded", "render_sharded", "allreduce_sum", "gather_screen"]


def ray_shards(nsamples, world, layout="strided"):
    """Sorted slots 0..n-1 of rays with per-ray sample counts `nsamples` dealt to `world` ranks.
    Returns one int64 array of slots per rank (ascending). "contiguous": rank r gets the slots whose
    sample prefix sum lies in (r total / world, (r + 1) total / world], so every shard's sample sum is
    within max(nsamples) of total / world. "strided": slot j goes to rank j mod world."""
    world = int(world)
    if world < 1:
        raise ValueError("world must be at least 1")
    ns = np.asarray(nsamples, dtype=np.int64).ravel()
    if ns.size and ns.min() < 0:
        raise ValueError("sample counts must be non-negative")
    n = ns.size
    if layout == "strided":
        return [np.arange(r, n, world, dtype=np.int64) for r in range(world)]
    if layout != "contiguous":
        raise ValueError(f"unknown layout {layout!r}")
    c = np.cumsum(ns)
    total = int(c[-1]) if n else 0
    # bound r: the number of rays whose prefix sum is at most r total / world (exact in integers)
    bounds = [0]
    for r in range(1, world):
        bounds.append(int(np.searchsorted(c * world, r * total, side="right")))
    bounds.append(n)
    return [np.arange(bounds[r], bounds[r + 1], dtype=np.int64) for r in range(world)]


def _world(group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


class RayShard:
    """This rank's rays of `camera` at spin `a`, inclination `theta_o`: `pixels` are their screen
    indices (ascending), `cache` a GeodesicCache regenerated on them alone (None for an empty shard),
    `pixels_by_rank` every rank's pixels. The whole screen is regenerated once, on this rank, to read
    the sorted order and the sample counts that the partition follows (regenerate! is deterministic,
    so every rank reads the same)."""

    def __init__(self, camera, nsamples, a, theta_o, rank=None, world=None, layout="strided", marcher=None, uneven=None,
                 device=0, group=None):
        if rank is None or world is None:
            r, w = _world(group)
            rank = r if rank is None else rank
            world = w if world is None else world
        if not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside a world of {world}")
        full = GeodesicCache(camera, nsamples, device)
        try:
            regenerate(full, a, theta_o, marcher=marcher, uneven=uneven)
            perm, counts = full.perm, full.nsamples_per_ray
        finally:
            full.close()
        slots = ray_shards(counts, world, layout)
        self.rank, self.world, self.layout = int(rank), int(world), layout
        self.npix_full = camera.npix
        self.pixels_by_rank = [np.sort(perm[s]) for s in slots]
        self.samples_by_rank = [int(counts[s].sum()) for s in slots]
        self.pixels = self.pixels_by_rank[rank]
        self.cache = None
        if self.pixels.size:
            self.cache = GeodesicCache(Camera(camera.alpha[self.pixels], camera.beta[self.pixels]), nsamples, device)
            regenerate(self.cache, a, theta_o, marcher=marcher, uneven=uneven)
        self._index = {}

    def take(self, x, axis):
        """This rank's pixels of a screen-order array (numpy or torch) along `axis`. A CUDA tensor is
        gathered on torch's current stream, which is waited for: the library reads its inputs on
        its own stream."""
        if hasattr(x, "data_ptr"):
            import torch
            key = str(x.device)
            if key not in self._index:
                self._index[key] = torch.as_tensor(self.pixels, device=x.device)
            out = x.index_select(axis, self._index[key]).contiguous()
            if out.is_cuda:
                torch.cuda.current_stream(out.device).synchronize()
            return out
        return np.ascontiguousarray(np.take(x, self.pixels, axis=axis))

    def close(self):
        if self.cache is not None:
            self.cache.close()
            self.cache = None


def _nparams(model):
    return sum(_lib.NROWS[s.kind] * s.nsplat for s in model.sets())


def _split(model, flat):
    out, q = [], 0
    for s in model.sets():
        nr = _lib.NROWS[s.kind]
        out.append(np.asarray(flat[q:q + nr * s.nsplat]).reshape(s.nsplat, nr).T.copy())
        q += nr * s.nsplat
    return out[0] if len(out) == 1 else out


def allreduce_sum(vec, group=None):
    """SUM all-reduce of a float64 vector over the ranks of `group` (identity without a process
    group or with one rank). NCCL reduces a copy on this rank's GPU; gloo the host copy."""
    import torch
    import torch.distributed as dist
    _, world = _world(group)
    v = np.ascontiguousarray(vec, dtype=np.float64)
    if world == 1:
        return v.copy()
    t = torch.from_numpy(v.copy())
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def chi2_gradient_shard(shard, model, times, nus, L, data, sigma, mask=None, nmax=-1, slab=0.0, precision=KS_MIXED):
    """chi^2 and its flat gradient over this rank's rays alone: [chi^2, dparams...] as one float64
    vector (dparams in the parameters' flat layout). `data`, `sigma` (unless scalar) and `mask` are
    the whole screen's arrays in screen order; each rank reads its own pixels."""
    vec = np.zeros(1 + _nparams(model))
    if shard.cache is None:
        return vec
    d = shard.take(data, 2)
    sg = sigma if np.isscalar(sigma) else shard.take(sigma, 2)
    mk = None if mask is None else shard.take(mask, 2)
    grad = vec[1:]
    chi2, _ = chi2_gradient(shard.cache, model, times, nus, L, d, sg, mask=mk, nmax=nmax, slab=slab, precision=precision,
                            dparams=grad)
    vec[0] = chi2
    return vec


def chi2_gradient_sharded(shard, model, times, nus, L, data, sigma, mask=None, nmax=-1, slab=0.0, precision=KS_MIXED,
                          group=None):
    """chi2_gradient! (Fit.jl:502-534) of the whole screen with each rank evaluating its own rays and
    one all-reduce: every rank returns (chi^2, grad), grad as chi2_gradient returns it."""
    vec = allreduce_sum(chi2_gradient_shard(shard, model, times, nus, L, data, sigma, mask=mask, nmax=nmax, slab=slab,
                                            precision=precision), group)
    return float(vec[0]), _split(model, vec[1:])


def gather_screen(pixels_by_rank, part, npix, group=None):
    """The whole screen from every rank's part: `part` is (..., len(pixels_by_rank[rank]), 4) on this
    rank; returns the (..., npix, 4) float64 screen-order array on every rank. The parts are padded to
    the largest shard for one all_gather."""
    import torch
    import torch.distributed as dist
    rank, world = _world(group)
    p = np.asarray(part.cpu() if hasattr(part, "data_ptr") else part, dtype=np.float64)
    lead = p.shape[:-2]
    out = np.zeros(lead + (npix, p.shape[-1]))
    if world == 1:
        out[..., pixels_by_rank[0], :] = p
        return out
    width = max(len(px) for px in pixels_by_rank)
    pad = np.zeros(lead + (width, p.shape[-1]))
    pad[..., :p.shape[-2], :] = p
    t = torch.from_numpy(pad)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    for r, px in enumerate(pixels_by_rank):
        out[..., px, :] = parts[r].cpu().numpy()[..., :len(px), :]
    return out


def render_sharded(shard, model, times, nus, L, nmax=-1, slab=0.0, precision=KS_MIXED, group=None):
    """render (polarized_cube) of the whole screen with each rank rendering its own rays: the
    (nfreq, nframes, npix, 4) screen-order image on every rank."""
    nt = int(np.atleast_1d(times).shape[0]) if not hasattr(times, "data_ptr") else int(times.shape[0])
    nf = int(np.atleast_1d(nus).shape[0]) if not hasattr(nus, "data_ptr") else int(nus.shape[0])
    if shard.cache is None:
        part = np.zeros((nf, nt, 0, 4))
    else:
        part = render(shard.cache, model, times, nus, L, nmax=nmax, slab=slab, precision=precision)
    return gather_screen(shard.pixels_by_rank, part, shard.npix_full, group)
