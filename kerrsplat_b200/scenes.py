"""Seeded synthetic scenes of the five benchmark configurations (numpy PCG64 draws).

The reference publishes no scene files for these workloads; these generators stand in for them
with the shapes, sizes and value distributions of each configuration. Parameter matrices use the
reference's row layouts (Splats.jl:54, polarized.jl:17-19, populations.jl:13-26), one column per
splat.
"""
import numpy as np

from . import Camera, gravitational_radius


def _geometry(rng, n, rlo, rhi, a, theta_range=(np.pi / 3, 2 * np.pi / 3)):
    r = rng.uniform(rlo, rhi, n)
    th = rng.uniform(*theta_range, n)
    ph = rng.uniform(0.0, 2 * np.pi, n)
    xyz = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)])
    widths = np.exp(rng.uniform(np.log(0.3), np.log(2.0), (3, n)))
    q = rng.standard_normal((4, n))
    q /= np.linalg.norm(q, axis=0)
    omega = 1.0 / (r ** 1.5 + a)
    return r, th, xyz, np.log(widths), q, omega


def keplerian_zamo_velocity(a, r, th):
    """ZAMO-frame spatial 4-velocity of the prograde circular orbit Omega = 1/(r^(3/2) + a)
    (Fit.jl:786-796), with the Boyer-Lindquist metric and the ZAMO tetrad (t, r, phi, -theta)."""
    s2 = np.sin(th) ** 2
    Sg = r * r + a * a * np.cos(th) ** 2
    D = r * r - 2 * r + a * a
    A = (r * r + a * a) ** 2 - a * a * D * s2
    gtt = -(1 - 2 * r / Sg)
    gtp = -2 * a * r * s2 / Sg
    gpp = A * s2 / Sg
    Om = 1.0 / (r * np.sqrt(r) + a)
    ut2 = -(gtt + 2 * gtp * Om + gpp * Om * Om)
    ut = 1.0 / np.sqrt(np.maximum(ut2, np.finfo(float).eps))
    lapse = np.sqrt(Sg * D / A)
    om = 2 * a * r / A
    varpi = np.sqrt(A / Sg) * np.sqrt(s2)
    # u_zamo = (lapse ut, 0, varpi (ut Om - om ut), 0)
    return np.stack([np.zeros_like(r), varpi * (ut * Om - om * ut), np.zeros_like(r)])


def config1(res=128, N=512):
    """Thin image: a = 0.94, theta_o = 17 deg, +-15 M, N = 512, 12 THIN14 splats, seed 0."""
    rng = np.random.Generator(np.random.PCG64(0))
    a, tho, n = 0.94, np.deg2rad(17.0), 12
    r, th, xyz, s, q, om = _geometry(rng, n, 3.0, 10.0, a)
    p = np.zeros((14, n))
    p[0:3] = xyz; p[3:6] = s; p[6:10] = q
    p[10] = 0.0; p[11] = np.log(1e9)
    p[12] = rng.uniform(0.0, np.log(10.0), n)
    p[13] = om
    return dict(a=a, theta_o=tho, camera=Camera((-15.0, 15.0), (-15.0, 15.0), res), N=N, M=64, params=p, t_obs=0.0, nu=230e9)


def thermal_params(rng, n, a, rlo=2.5, rhi=12.0):
    r, th, xyz, s, q, om = _geometry(rng, n, rlo, rhi, a)
    p = np.zeros((21, n))
    p[0:3] = xyz; p[3:6] = s; p[6:10] = q
    p[10] = 0.0; p[11] = np.log(1e9)
    p[12] = np.log(np.exp(rng.uniform(np.log(1e4), np.log(1e6), n)))
    p[13] = np.log(np.exp(rng.uniform(np.log(1.0), np.log(50.0), n)))
    p[14] = np.log(rng.uniform(1.0, 30.0, n))
    p[15] = np.arccos(rng.uniform(-1.0, 1.0, n))
    p[16] = rng.uniform(0.0, 2 * np.pi, n)
    uk = keplerian_zamo_velocity(a, r, th)
    nrm = np.linalg.norm(uk, axis=0)
    p[17:20] = uk + 0.1 * nrm * rng.standard_normal((3, n))
    p[20] = om
    return p


def config2(res=256, N=1024):
    """Polarized image: a = 0.5, theta_o = 60 deg, +-20 M, N = 1024, 64 THERMAL21 splats at
    86, 230, 345 GHz, seed 1."""
    rng = np.random.Generator(np.random.PCG64(1))
    a, tho = 0.5, np.deg2rad(60.0)
    p = thermal_params(rng, 64, a)
    return dict(a=a, theta_o=tho, camera=Camera((-20.0, 20.0), (-20.0, 20.0), res), N=N, M=64, params=p,
                t_obs=0.0, nus=np.array([86e9, 230e9, 345e9]), L=gravitational_radius(4.0e6))


def _population_rows(rng, n, a, rlo=2.5, rhi=12.0):
    """The 22-row layout shared by power-law and kappa splats (populations.jl:13-26) with the
    geometry, field and velocity rows of thermal_params; rows 13-14 are set by the caller."""
    r, th, xyz, s, q, om = _geometry(rng, n, rlo, rhi, a)
    p = np.zeros((22, n))
    p[0:3] = xyz; p[3:6] = s; p[6:10] = q
    p[10] = 0.0; p[11] = np.log(1e9)
    p[12] = np.log(np.exp(rng.uniform(np.log(1e4), np.log(1e6), n)))
    p[15] = np.log(rng.uniform(1.0, 30.0, n))
    p[16] = np.arccos(rng.uniform(-1.0, 1.0, n))
    p[17] = rng.uniform(0.0, 2 * np.pi, n)
    uk = keplerian_zamo_velocity(a, r, th)
    nrm = np.linalg.norm(uk, axis=0)
    p[18:21] = uk + 0.1 * nrm * rng.standard_normal((3, n))
    p[21] = om
    return p


def powerlaw_params(rng, n, a):
    """Power-law splats: p ~ U[2.5, 3.5], gamma_min = 10 (populations.jl:13-15)."""
    p = _population_rows(rng, n, a)
    p[13] = rng.uniform(2.5, 3.5, n)
    p[14] = np.log(10.0)
    return p


def kappa_params(rng, n, a):
    """kappa splats: kappa ~ U[3, 6], w = log-uniform in [1, 50] (populations.jl:24-26)."""
    p = _population_rows(rng, n, a)
    p[13] = rng.uniform(3.0, 6.0, n)
    p[14] = np.log(np.exp(rng.uniform(np.log(1.0), np.log(50.0), n)))
    return p


def config3_target(params, rng_seed=2):
    """The perturbed parameters of the configuration-3 target: every parameter moved by 5% Gaussian
    noise relative to max(|p|, 0.1); the caller renders them and adds 1% Gaussian pixel noise
    (sigma = 0.01 max I)."""
    rng = np.random.Generator(np.random.PCG64(rng_seed))
    return params + 0.05 * np.maximum(np.abs(params), 0.1) * rng.standard_normal(params.shape), rng
