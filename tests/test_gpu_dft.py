"""The image-to-visibility DFT, its adjoint and the frame chi^2 + seed (device_visibilities.jl)
against the numpy FP64 restatement in the oracle: the FP64 direct path to 1e-10, the 3xTF32
tensor-core path to FP32 accuracy (1e-5 relative), and the adjoint identity <seed, I> = Re <w, V(I)>."""
import numpy as np
import pytest

import kerrsplat_b200 as ks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dft_case():
    na, nb = 48, 40
    cam = ks.Camera((-16.0, 16.0), (-14.0, 14.0), (na, nb))
    cache = ks.GeodesicCache(cam, 8)
    ks.regenerate(cache, 0.7, np.deg2rad(30.0))
    rng = np.random.Generator(np.random.PCG64(4))
    img = np.abs(rng.standard_normal((na * nb, 4))) * np.array([1.0, 0.2, 0.2, 0.05])
    nuv = 300
    rad = 10e9 * np.sqrt(rng.uniform(0, 1, nuv))
    ang = rng.uniform(0, 2 * np.pi, nuv)
    u, v = rad * np.cos(ang), rad * np.sin(ang)
    L, D = ks.gravitational_radius(6.5e9), 16.8e6 * 3.085678e18
    psize = (32.0 / (na - 1)) * L / D
    scale = psize ** 2 / 1e-23
    tap = np.exp(-rng.uniform(0, 0.3, nuv))
    return dict(cache=cache, na=na, nb=nb, img=img, u=u, v=v, psize=psize, scale=scale, tap=tap, rng=rng)


def rel(x, y):
    return np.linalg.norm(x - y) / np.linalg.norm(y)


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-5)])
def test_visibilities_match_oracle(dft_case, oracle, prec, tol):
    c = dft_case
    ref = oracle.visibilities(c["img"], c["na"], c["nb"], c["u"], c["v"], c["tap"], c["psize"], c["scale"])
    got = ks.visibilities(c["cache"], c["img"], c["u"], c["v"], c["psize"], c["scale"], tap=c["tap"], precision=prec)
    assert rel(got, ref) < tol, rel(got, ref)
    # sorted-order input gives the same visibilities
    perm = c["cache"].perm
    got_s = ks.visibilities(c["cache"], c["img"][perm], c["u"], c["v"], c["psize"], c["scale"], tap=c["tap"], precision=prec, order="sorted")
    assert rel(got_s, ref) < tol


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 1e-10), (ks.KS_MIXED, 1e-5)])
def test_seed_and_chi2_match_oracle(dft_case, oracle, prec, tol):
    c = dft_case
    rng = c["rng"]
    nuv = c["u"].size
    w = rng.standard_normal((nuv, 4)) + 1j * rng.standard_normal((nuv, 4))
    ref = oracle.vis_seed(w, c["na"], c["nb"], c["u"], c["v"], c["tap"], c["psize"], c["scale"])
    got = ks.vis_seed(c["cache"], w, c["u"], c["v"], c["psize"], c["scale"], tap=c["tap"], precision=prec)
    assert rel(got, ref) < tol, rel(got, ref)
    # adjoint identity
    V = ks.visibilities(c["cache"], c["img"], c["u"], c["v"], c["psize"], c["scale"], tap=c["tap"], precision=prec)
    lhs = np.sum(got * c["img"])
    rhs = np.sum(np.real(w * np.conj(V)))
    assert abs(lhs - rhs) < tol * max(abs(rhs), 1.0) * 10
    # chi^2 and its seed, with gains
    Vt = oracle.visibilities(c["img"] * 1.05, c["na"], c["nb"], c["u"], c["v"], c["tap"], c["psize"], c["scale"])
    # thermal-noise-like sigma: one value per Stokes parameter, 5% of its rms amplitude (a sigma that
    # follows |V| of every baseline would amplify the FP32 forward error of the weakest ones)
    sigma = np.broadcast_to(0.05 * np.sqrt(np.mean(np.abs(Vt) ** 2, axis=0)), Vt.shape).copy()
    gains = np.exp(1j * rng.uniform(-0.1, 0.1, nuv)) * rng.uniform(0.9, 1.1, nuv)
    x_ref, s_ref = oracle.frame_chi2_seed(c["img"], c["na"], c["nb"], c["u"], c["v"], c["tap"], gains, Vt, sigma, c["psize"], c["scale"])
    x, s = ks.frame_chi2_seed(c["cache"], c["img"], c["u"], c["v"], Vt, sigma, c["psize"], c["scale"], tap=c["tap"], gains=gains, precision=prec)
    assert abs(x - x_ref) / x_ref < tol * 10
    assert rel(s, s_ref) < tol * 10


@pytest.mark.parametrize("prec,tol", [(ks.KS_FP64, 5e-7), (ks.KS_MIXED, 2e-5)])
def test_transform_of_ehtim_source_image_matches_its_observation(prec, tol):
    """The GPU transform (FP64 direct and 3xTF32) of the ehtim observation's source image against the
    observation's noiseless visibilities (the sky conventions, east = -alpha, pinned against an
    independent code: test/test_uvfits.jl), in Jy with scale 1."""
    import os
    from kerrsplat_b200 import fitsio
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "uvfits")
    img, hdr = fitsio.read_stokes_fits(os.path.join(d, "synth_eht2017_image.fits"))
    psize = hdr["psize_deg"] * np.pi / 180
    clean = fitsio.read_uvfits(os.path.join(d, "synth_eht2017_noiseless.uvfits"))
    cam = ks.Camera((-16.0, 16.0), (-16.0, 16.0), 32)
    cache = ks.GeodesicCache(cam, 8)
    ks.regenerate(cache, 0.5, np.deg2rad(30.0))
    V = ks.visibilities(cache, img.reshape(32 * 32, 4, order="F"), clean.u, clean.v, psize, 1.0, precision=prec)
    err = np.max(np.abs(V - clean.vis))
    print("GPU transform of the source image vs the noiseless observation", prec, err)
    assert err < tol
    cache.close()
