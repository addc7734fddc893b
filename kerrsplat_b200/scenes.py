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


# ---- trajectory knots (host preprocessing, trajectories.jl:9-68) ------------------------------------

def boyer_lindquist(a, x, y, z):
    """BL (r, theta, phi) of a quasi-Cartesian Kerr-Schild point (trajectories.jl:9-18)."""
    r = np.sqrt(x * x + y * y + z * z)
    th = np.arccos(np.clip(z / r, -1.0, 1.0))
    temp = np.sqrt(1 - a * a)
    rp, rm = 1 + temp, 1 - temp
    eps = np.finfo(float).eps
    phks = np.arctan2(y, x)
    ph = phks - a / (2 * temp) * np.log(np.abs((r - rp + eps) / (r - rm + eps))) + np.arctan2(a, r)
    return r, th, ph


def quasi_cartesian_kerr_schild(a, r, th, ph):
    """coordinates.jl:22-31."""
    temp = np.sqrt(1 - a * a)
    rp, rm = 1 + temp, 1 - temp
    eps = np.finfo(float).eps
    phks = ph + a / (2 * temp) * np.log(np.abs((r - rp + eps) / (r - rm + eps))) - np.arctan2(a, r)
    return r * np.sin(th) * np.cos(phks), r * np.sin(th) * np.sin(phks), r * np.cos(th)


def coordinate_velocity(a, r, th, u):
    """(dr/dt, dtheta/dt, dphi/dt) of ZAMO 3-velocity u along (r-hat, phi-hat, -theta-hat)
    (trajectories.jl:21-25): the BL 4-velocity from the ZAMO tetrad."""
    g = np.sqrt(1 + u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    s2 = np.sin(th) ** 2
    Sg = r * r + a * a * np.cos(th) ** 2
    D = r * r - 2 * r + a * a
    A = (r * r + a * a) ** 2 - a * a * D * s2
    lapse = np.sqrt(Sg * D / A)
    om = 2 * a * r / A
    varpi = np.sqrt(A / Sg) * np.sqrt(s2)
    ut = g / lapse
    ur = np.sqrt(D / Sg) * u[0]
    uth = -u[2] / np.sqrt(Sg)
    uph = om / lapse * g + u[1] / varpi
    return np.array([ur / ut, uth / ut, uph / ut])


def trajectory_knots(params, a, times, substeps=4):
    """Centres of every splat at the coordinate `times`, integrated from the centre at t0 with the
    splat's ZAMO velocity by RK4 in BL coordinates, `substeps` steps per knot interval, forward and
    backward from t0 (trajectories.jl:35-68). Returns (3, nknots, nsplat) KS positions."""
    times = np.asarray(times, dtype=np.float64)
    n = params.shape[1]
    knots = np.empty((3, times.size, n))
    dt_knot = abs(times[-1] - times[0]) / max(times.size - 1, 1)
    for i in range(n):
        u = params[17:20, i]
        t0 = params[10, i]
        q0 = np.array(boyer_lindquist(a, *params[0:3, i]))

        def integrate(q, t_from, t_to):
            m = max(1, int(np.ceil(abs(t_to - t_from) / dt_knot * substeps)))
            h = (t_to - t_from) / m
            for _ in range(m):
                k1 = coordinate_velocity(a, q[0], q[1], u)
                k2 = coordinate_velocity(a, *(q + h / 2 * k1)[:2], u)
                k3 = coordinate_velocity(a, *(q + h / 2 * k2)[:2], u)
                k4 = coordinate_velocity(a, *(q + h * k3)[:2], u)
                q = q + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
            return q

        order = np.argsort(times)
        kt0 = int(np.searchsorted(times[order], t0))
        q, tprev = q0, t0
        for k in range(kt0, times.size):
            q = integrate(q, tprev, times[order[k]]); tprev = times[order[k]]
            knots[:, order[k], i] = quasi_cartesian_kerr_schild(a, *q)
        q, tprev = q0, t0
        for k in range(kt0 - 1, -1, -1):
            q = integrate(q, tprev, times[order[k]]); tprev = times[order[k]]
            knots[:, order[k], i] = quasi_cartesian_kerr_schild(a, *q)
    return knots


def config4(res=512, N=2048, nframes=32, density=768.0, nmin=128):
    """Batched movie: a = 0.94, theta_o = 163 deg, +-15 M, frames t_obs = 10 f M (f < nframes),
    86/230/345/690 GHz, uneven samples per ray (N_j = clamp(64 ceil(768 tau_j / 64), 128, 2048)),
    256 splats of seed 3: 85 thermal on 4 trajectory knots spanning the emission times, 85 power-law
    (p ~ U[2.5, 3.5], gamma_min = 10), 86 kappa (kappa ~ U[3, 6])."""
    rng = np.random.Generator(np.random.PCG64(3))
    a, tho = 0.94, np.deg2rad(163.0)
    pt = thermal_params(rng, 85, a)
    pp = powerlaw_params(rng, 85, a)
    pk = kappa_params(rng, 86, a)
    times = 10.0 * np.arange(nframes)
    # knots over the emission times of the movie: lookbacks reach ~ -60 M before the first frame
    ktimes = np.linspace(times[0] - 80.0, times[-1] + 20.0, 4)
    knots = trajectory_knots(pt, a, ktimes)
    return dict(a=a, theta_o=tho, camera=Camera((-15.0, 15.0), (-15.0, 15.0), res), N=N, M=64, density=density, nmin=nmin,
                thermal=pt, powerlaw=pp, kappa=pk, knots=knots, knot_times=ktimes, times=times,
                nus=np.array([86e9, 230e9, 345e9, 690e9]), L=gravitational_radius(4.0e6))


def config5(res=1024, N=512, nsets=16, nuv=2000):
    """Minibatched fit: a = 0.7, theta_o = 30 deg, +-16 M, N = 512 (assumed), 230 GHz, seed 4; nsets
    THERMAL21 sets with S ~ U{32..512} splats; nuv (u, v) points uniform in a disk of radius 10 G-lambda;
    M = 6.5e9 Msun, D = 16.8 Mpc (pixel size psize = d(alpha) L / D); the target of each set is its own
    scene with every parameter perturbed by 5% (config-3 rule), observed with 2% complex Gaussian noise
    relative to |V| (sigma = 0.02 |V|, floored at 1e-3 of the largest |V|)."""
    rng = np.random.Generator(np.random.PCG64(4))
    a, tho = 0.7, np.deg2rad(30.0)
    counts = rng.integers(32, 513, nsets)
    sets = [thermal_params(rng, int(s), a) for s in counts]
    rad = 10e9 * np.sqrt(rng.uniform(0.0, 1.0, nuv))
    ang = rng.uniform(0.0, 2 * np.pi, nuv)
    L = gravitational_radius(6.5e9)
    D = 16.8e6 * 3.0857e18
    dalpha = 32.0 / (res - 1)
    psize = dalpha * L / D
    return dict(a=a, theta_o=tho, camera=Camera((-16.0, 16.0), (-16.0, 16.0), res), N=N, M=64, sets=sets, counts=counts,
                u=rad * np.cos(ang), v=rad * np.sin(ang), psize=psize, scale=psize ** 2 / 1e-23, L=L, nu=230e9, t_obs=0.0, rng=rng)
