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


def _ragged_case(na, nb, nuv, seed):
    cam = ks.Camera((-16.0, 16.0), (-14.0, 14.0), (na, nb))
    cache = ks.GeodesicCache(cam, 8)
    ks.regenerate(cache, 0.7, np.deg2rad(30.0))
    rng = np.random.Generator(np.random.PCG64(seed))
    img = np.abs(rng.standard_normal((na * nb, 4))) * np.array([1.0, 0.2, 0.2, 0.05])
    rad = 10e9 * np.sqrt(rng.uniform(0, 1, nuv))
    ang = rng.uniform(0, 2 * np.pi, nuv)
    L, D = ks.gravitational_radius(6.5e9), 16.8e6 * 3.085678e18
    psize = (32.0 / max(na - 1, 1)) * L / D
    w = rng.standard_normal((nuv, 4)) + 1j * rng.standard_normal((nuv, 4))
    return cache, img, rad * np.cos(ang), rad * np.sin(ang), psize, psize ** 2 / 1e-23, np.exp(-rng.uniform(0, 0.3, nuv)), w


@pytest.mark.parametrize("na,nb,nuv", [(48, 40, 300), (37, 29, 131), (130, 3, 1), (8, 200, 257), (300, 33, 70)])
def test_tensor_paths_agree_on_ragged_shapes(oracle, na, nb, nuv):
    """The tcgen05 GEMM (TMA tiles, UMMA into TMEM) and the mma.sync fallback on the same split
    operands, at shapes with partial tiles in M, N and K (K = na < 32, na not a multiple of 4, one
    baseline): both within 1e-5 of the FP64 oracle (forward and adjoint) and within 1e-6 of each other
    (they differ only in the FP32 accumulation order)."""
    cache, img, u, v, psize, scale, tap, w = _ragged_case(na, nb, nuv, 7 + na)
    ref_v = oracle.visibilities(img, na, nb, u, v, tap, psize, scale)
    ref_s = oracle.vis_seed(w, na, nb, u, v, tap, psize, scale)
    got = {}
    for path in ("tcgen05", "mma.sync"):
        cache.set_tensor_path(path)
        got[path] = (ks.visibilities(cache, img, u, v, psize, scale, tap=tap, precision=ks.KS_MIXED),
                     ks.vis_seed(cache, w, u, v, psize, scale, tap=tap, precision=ks.KS_MIXED))
        assert rel(got[path][0], ref_v) < 1e-5, (path, rel(got[path][0], ref_v))
        assert rel(got[path][1], ref_s) < 1e-5, (path, rel(got[path][1], ref_s))
    cache.set_tensor_path("tcgen05")
    assert rel(got["tcgen05"][0], got["mma.sync"][0]) < 1e-6
    assert rel(got["tcgen05"][1], got["mma.sync"][1]) < 1e-6
    # repeated calls are bitwise reproducible (fixed tiles, fixed accumulation order)
    again = ks.visibilities(cache, img, u, v, psize, scale, tap=tap, precision=ks.KS_MIXED)
    assert np.array_equal(again, got["tcgen05"][0])
    cache.close()


@pytest.mark.parametrize("m,n", [(1000, 77), (131, 300), (5, 3)])
def test_normal_matrix_tensor_paths(m, n):
    """J^T J through both GEMM kernels (Jt Jt^T from one split transposed copy) against numpy. The
    bound is 5e-5 of the largest entry: the products are 3xTF32-exact to ~5e-7, and what remains is the
    FP32 accumulation of K = m terms in the tensor cores (up to m 2^-23 relative for same-sign terms,
    1.1e-5 measured at m = 1000); both kernels accumulate in the same order and agree to 1e-6."""
    cam = ks.Camera((-1.0, 1.0), (-1.0, 1.0), 2)
    cache = ks.GeodesicCache(cam, 8)
    rng = np.random.Generator(np.random.PCG64(m + n))
    J = rng.standard_normal((m, n)) * np.exp(rng.uniform(-2, 2, n))[None]
    ref = J.T @ J
    out = {}
    for path in ("tcgen05", "mma.sync"):
        cache.set_tensor_path(path)
        out[path] = ks.normal_matrix(cache, J, precision=ks.KS_MIXED)
        assert np.max(np.abs(out[path] - ref)) <= 5e-5 * np.abs(ref).max(), path
    assert np.max(np.abs(out["tcgen05"] - out["mma.sync"])) <= 1e-6 * np.abs(ref).max()
    cache.close()


def test_tensor_core_gemm_wait_gives_up_cleanly():
    """The tcgen05 GEMM's bounded waits: under the test hook its operand barriers are armed but no
    tile copy is issued, every wait gives up after ~10 ms, the blocks free their TMEM and return, and
    the call fails with KS_ERR_TIMEOUT; the context then computes the same visibilities as before."""
    cache, img, u, v, psize, scale, tap, w = _ragged_case(40, 36, 200, 3)
    ref = ks.visibilities(cache, img, u, v, psize, scale, tap=tap, precision=ks.KS_MIXED)
    cache.set_stage_test(True)
    with pytest.raises(ks.KsError) as err:
        ks.visibilities(cache, img, u, v, psize, scale, tap=tap, precision=ks.KS_MIXED)
    assert err.value.status == ks._lib.KS_ERR_TIMEOUT
    cache.set_stage_test(False)
    again = ks.visibilities(cache, img, u, v, psize, scale, tap=tap, precision=ks.KS_MIXED)
    assert np.array_equal(again, ref)
    cache.close()
