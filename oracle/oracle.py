"""ctypes binding of the CPU oracle (oracle/_build/libks_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, never by the kerrsplat_b200 package. `build()` compiles it with the Makefile beside this file.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libks_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.kso_num_threads.restype = ctypes.c_int
    return _lib


def _p(x):
    return ctypes.c_void_p(x.ctypes.data)


def _d(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def set_threads(n):
    load().kso_set_num_threads(int(n))


def num_threads():
    return load().kso_num_threads()


def ray_constants(a, theta_o, alpha, beta):
    alpha, beta = _d(alpha), _d(beta)
    out = np.empty((alpha.size, 24))
    load().kso_ray_constants(ctypes.c_double(a), ctypes.c_double(theta_o), _p(alpha), _p(beta), ctypes.c_long(alpha.size), _p(out))
    return out


def march_samples(a, theta_o, alpha, beta, N, M=64):
    """Sample stream of the recurrence march: dict of (npix, N) arrays, screen order."""
    alpha, beta = _d(alpha), _d(beta)
    n = alpha.size
    t, r, th, ph = (np.empty((n, N)) for _ in range(4))
    fl = np.empty((n, N), dtype=np.uint8)
    rt, rp = np.empty(n), np.empty(n)
    load().kso_march_samples(ctypes.c_double(a), ctypes.c_double(theta_o), _p(alpha), _p(beta), ctypes.c_long(n), int(N), int(M),
                             _p(t), _p(r), _p(th), _p(ph), _p(fl), _p(rt), _p(rp))
    return {"t": t, "r": r, "theta": th, "phi": ph, "flags": fl, "resid_t": rt, "resid_phi": rp}


def anchor_values(a, theta_o, alpha, beta, N):
    """t~ and phi of the anchor evaluator at every sample (no recurrence): (npix, N) arrays."""
    alpha, beta = _d(alpha), _d(beta)
    n = alpha.size
    t, ph = np.empty((n, N)), np.empty((n, N))
    ok = np.empty((n, N), dtype=np.uint8)
    load().kso_anchor_values(ctypes.c_double(a), ctypes.c_double(theta_o), _p(alpha), _p(beta), ctypes.c_long(n), int(N), _p(t), _p(ph), _p(ok))
    return t, ph, ok


def thin_image(a, theta_o, alpha, beta, N, M, params, t_obs):
    alpha, beta = _d(alpha), _d(beta)
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).T)
    n = alpha.size
    out, rt, rp = np.empty(n), np.empty(n), np.empty(n)
    load().kso_thin_image(ctypes.c_double(a), ctypes.c_double(theta_o), _p(alpha), _p(beta), ctypes.c_long(n), int(N), int(M),
                          _p(p), int(p.shape[0]), ctypes.c_double(t_obs), _p(out), _p(rt), _p(rp))
    return out


KIND = {"thermal": 1, "powerlaw": 2, "kappa": 3, "knot": 4}
NROWS = {1: 21, 2: 22, 3: 22, 4: 21}


def polarized_image(a, theta_o, alpha, beta, N, M, sets, t_obs, nu, L, nmax=-1, slab=0.0, gmax=1e5):
    """sets: list of (kind, params (nrows, nsplat), hyp or None[, knots (3, nknots, nsplat), knot_times]).
    Returns (npix, 4) cgs, screen order."""
    alpha, beta = _d(alpha), _d(beta)
    n = alpha.size
    ns = len(sets)
    kinds = (ctypes.c_int * ns)(*[KIND[st[0]] if isinstance(st[0], str) else st[0] for st in sets])
    nrows = (ctypes.c_int * ns)(*[NROWS[kinds[i]] for i in range(ns)])
    keep = [np.ascontiguousarray(np.asarray(st[1], dtype=np.float64).T) for st in sets]
    nsplat = (ctypes.c_int * ns)(*[k.shape[0] for k in keep])
    params = (ctypes.c_void_p * ns)(*[k.ctypes.data for k in keep])
    hyps = [None if st[2] is None else _d(st[2]) for st in sets]
    hyp = (ctypes.c_void_p * ns)(*[None if h is None else h.ctypes.data for h in hyps])
    # knots (3, nknots, nsplat) in the reference's column-major order: x fastest
    kn = [np.asfortranarray(np.asarray(st[3], dtype=np.float64)).ravel(order="F") if len(st) > 3 else None for st in sets]
    kt = [_d(st[4]) if len(st) > 4 else None for st in sets]
    knots = (ctypes.c_void_p * ns)(*[None if k is None else k.ctypes.data for k in kn])
    ktimes = (ctypes.c_void_p * ns)(*[None if k is None else k.ctypes.data for k in kt])
    nknots = (ctypes.c_int * ns)(*[0 if k is None else k.size for k in kt])
    out = np.empty((n, 4))
    load().kso_polarized_image(ctypes.c_double(a), ctypes.c_double(theta_o), _p(alpha), _p(beta), ctypes.c_long(n), int(N), int(M),
                               ns, kinds, nrows, nsplat, params, hyp, knots, ktimes, nknots, ctypes.c_double(gmax),
                               ctypes.c_double(t_obs), ctypes.c_double(nu), ctypes.c_double(L), int(nmax), ctypes.c_double(slab), _p(out))
    return out


def transfer_step(j, alpha, rho, D):
    O, E = np.empty(16), np.empty(4)
    j, alpha, rho = _d(j), _d(alpha), _d(rho)   # keep the buffers alive across the call
    load().kso_transfer_step(_p(j), _p(alpha), _p(rho), ctypes.c_double(D), _p(O), _p(E))
    return O.reshape(4, 4), E


def thermal(ne, Te, B, nu, th, dexter_rhoV=False, pandya=False):
    args = [_d(np.atleast_1d(x)) for x in (ne, Te, B, nu, th)]
    n = args[0].size
    out = np.empty((n, 8))
    load().kso_thermal(ctypes.c_long(n), *[_p(x) for x in args], int(dexter_rhoV), int(pandya), _p(out))
    return out


def riaf_image(a, theta_o, alpha, beta, N, M, nu, L, pandya=True, mirror_chi=False):
    """ipole's example RIAF (test/riaf_model.jl) through the polarized consumer: (npix, 4) cgs,
    screen order. `mirror_chi` plants a sign error in the screen angle (tests of the comparison)."""
    alpha, beta = _d(alpha), _d(beta)
    n = alpha.size
    out = np.empty((n, 4))
    load().kso_riaf_image(ctypes.c_double(a), ctypes.c_double(theta_o), _p(alpha), _p(beta), ctypes.c_long(n), int(N), int(M),
                          int(pandya), ctypes.c_double(nu), ctypes.c_double(L), int(mirror_chi), _p(out))
    return out


def powerlaw(ne, p, gmin, gmax, B, nu, th):
    args = [_d(np.atleast_1d(x)) for x in (ne, p, gmin, gmax, B, nu, th)]
    n = args[0].size
    out = np.empty((n, 8))
    load().kso_powerlaw(ctypes.c_long(n), *[_p(x) for x in args], _p(out))
    return out


def kappa(ne, kap, w, B, nu, th, hyp):
    args = [_d(np.atleast_1d(x)) for x in (ne, kap, w, B, nu, th, hyp)]
    n = args[0].size
    out = np.empty((n, 8))
    load().kso_kappa(ctypes.c_long(n), *[_p(x) for x in args], _p(out))
    return out


def besselk01(x):
    x = _d(np.atleast_1d(x))
    k0, k1 = np.empty_like(x), np.empty_like(x)
    load().kso_besselk01(ctypes.c_long(x.size), _p(x), _p(k0), _p(k1))
    return k0, k1


def jacobi_state(u, m):
    u, m = _d(np.atleast_1d(u)), _d(np.atleast_1d(m))
    sn, cn, dn = np.empty_like(u), np.empty_like(u), np.empty_like(u)
    load().kso_jacobi_state(ctypes.c_long(u.size), _p(u), _p(m), _p(sn), _p(cn), _p(dn))
    return sn, cn, dn


def ellipf(phi, m):
    phi, m = _d(np.atleast_1d(phi)), _d(np.atleast_1d(m))
    out = np.empty_like(phi)
    load().kso_ellipf(ctypes.c_long(phi.size), _p(phi), _p(m), _p(out))
    return out


# ---- visibilities: numpy FP64 restatement of src/Fit/device_visibilities.jl:53-111 ----------------

def pixel_offsets(na, nb, psize):
    """l (east is -alpha) and m of every screen pixel p = i + j na (device_visibilities.jl:53-58)."""
    i = np.arange(na * nb) % na
    j = np.arange(na * nb) // na
    return -((i + 1) - (na + 1) / 2) * psize, ((j + 1) - (nb + 1) / 2) * psize


def visibilities(image, na, nb, u, v, tap, psize, scale):
    """V_k = tap_k sum_j I_j scale exp(2 pi i (u_k l_j + v_k m_j)); image (npix, 4) in screen order
    (vis_kernel!, device_visibilities.jl:61-73). Returns (nuv, 4) complex."""
    l, m = pixel_offsets(na, nb, psize)
    ph = 2 * np.pi * (np.outer(u, l) + np.outer(v, m))
    E = np.exp(1j * ph) * scale
    V = E @ np.asarray(image, dtype=np.float64)
    return V * (np.ones(len(u)) if tap is None else np.asarray(tap))[:, None]


def vis_seed(w, na, nb, u, v, tap, psize, scale):
    """seed_j = sum_k Re[w_k conj(dV_k/dI_j)] (seed_kernel!, device_visibilities.jl:76-88); w (nuv, 4)
    complex. Returns (npix, 4) in screen order."""
    l, m = pixel_offsets(na, nb, psize)
    ph = 2 * np.pi * (np.outer(u, l) + np.outer(v, m))
    f = scale * (np.ones(len(u)) if tap is None else np.asarray(tap))
    E = np.exp(-1j * ph) * f[:, None]
    return np.real(E.T @ np.asarray(w))


def frame_chi2_seed(image, na, nb, u, v, tap, g, vis, sigma, psize, scale):
    """chi^2 of the gained model against the data and the adjoint seed (device_visibilities.jl:97-111)."""
    V = visibilities(image, na, nb, u, v, tap, psize, scale)
    gg = np.ones(len(u)) if g is None else np.asarray(g)
    r = (gg[:, None] * V - vis) / sigma
    w = 2 * np.conj(gg)[:, None] * r / sigma
    return float(np.sum(np.abs(r) ** 2)), vis_seed(w, na, nb, u, v, tap, psize, scale)
