"""The data formats either side of the path (kerrsplat_b200.fitsio; CPU only), pinned as the reference
pins its own readers (test/test_uvfits.jl): an ehtim-written polarized observation of the EHT 2017
array (tests/golden/uvfits/, copied from the reference's test/data by tests/golden/make_golden.py)
parsed row by row as ehtim parses it, and the direct transform of the observation's source image
(read by the FITS image reader) reproducing the noiseless visibilities to the float32 storage of the
file, which pins the transform's sky conventions (east = -alpha, north = +beta) against an
independent code; the noisy file gives a reduced chi^2 of one. Plus a write/read round trip of a
Stokes image."""
import csv
import os

import numpy as np
import pytest

from kerrsplat_b200 import fitsio

DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "uvfits")


def ehtim_csv(name):
    with open(os.path.join(DIR, name)) as f:
        rows = list(csv.DictReader(f))
    col = lambda k: np.array([float(r[k]) for r in rows])
    vis = np.stack([col(s + "re") + 1j * col(s + "im") for s in "IQUV"], axis=1)
    sig = np.stack([col("sig" + s) for s in "IQUV"], axis=1)
    return dict(time=col("time_h"), t1=[r["t1"].strip() for r in rows], t2=[r["t2"].strip() for r in rows], u=col("u"), v=col("v"),
                vis=vis, sigma=sig, tint=col("tint"))


@pytest.mark.parametrize("name", ["synth_eht2017", "synth_eht2017_noiseless"])
def test_uvfits_reader_matches_ehtim(name):
    obs = fitsio.read_uvfits(os.path.join(DIR, name + ".uvfits"))
    ref = ehtim_csv(name + "_ehtim.csv")
    assert len(obs) == len(ref["time"]) == 386
    assert obs.mjd == 57854 and obs.freq == 230e9 and obs.bandwidth == 1.856e9 and obs.source == "SYNTH"
    assert abs(obs.ra - 12.513728717168174) < 1e-9 and abs(obs.dec - 12.39112323919932) < 1e-9
    assert sorted(obs.stations) == ["AA", "AP", "AZ", "JC", "LM", "PV", "SM", "SR"]
    assert np.max(np.abs(obs.time - ref["time"])) < 1e-6
    assert [obs.stations[i] for i in obs.s1] == ref["t1"] and [obs.stations[i] for i in obs.s2] == ref["t2"]
    # ehtim multiplies the float32 UU, VV by the frequency in float32
    assert np.max(np.abs(obs.u - ref["u"]) / (np.abs(ref["u"]) + 1)) < 2e-7
    assert np.max(np.abs(obs.v - ref["v"]) / (np.abs(ref["v"]) + 1)) < 2e-7
    assert np.max(np.abs(obs.vis - ref["vis"])) < 1e-7
    assert np.max(np.abs(obs.sigma - ref["sigma"])) < 1e-9
    assert np.array_equal(obs.tint, ref["tint"])
    # the circular products are kept beside the Stokes visibilities
    assert np.allclose(obs.coh[:, 0], obs.vis[:, 0] + obs.vis[:, 3]) and np.allclose(obs.coh[:, 2], obs.vis[:, 1] + 1j * obs.vis[:, 2])
    pos = fitsio.antenna_positions(os.path.join(DIR, name + ".uvfits"))
    assert sorted(pos) == sorted(obs.stations) and all(p.shape == (3,) for p in pos.values())


def source_image():
    img, hdr = fitsio.read_stokes_fits(os.path.join(DIR, "synth_eht2017_image.fits"))
    psize = hdr["psize_deg"] * np.pi / 180
    return img, psize


def test_source_image_transform_matches_the_noiseless_observation(oracle):
    img, psize = source_image()
    assert img.shape == (32, 32, 4) and abs(psize - 200e-6 / 206264.806247 / 32) < 1e-13
    assert abs(img[..., 0].sum() - 1.4) < 1e-9
    clean = fitsio.read_uvfits(os.path.join(DIR, "synth_eht2017_noiseless.uvfits"))
    # pixel i + 32 j of the screen is image[i, j] (x, y); Jy/pixel in, Jy out (scale 1)
    flat = img.reshape(32 * 32, 4, order="F")
    model = oracle.visibilities(flat, 32, 32, clean.u, clean.v, None, psize, 1.0)
    err = np.max(np.abs(model - clean.vis))
    print("source image vs ehtim's noiseless visibilities:", err, "Jy")
    assert err < 5e-7
    mirrored = oracle.visibilities(img[::-1].reshape(32 * 32, 4, order="F"), 32, 32, clean.u, clean.v, None, psize, 1.0)
    assert np.max(np.abs(mirrored - clean.vis)) > 1e-2
    noisy = fitsio.read_uvfits(os.path.join(DIR, "synth_eht2017.uvfits"))
    m = oracle.visibilities(flat, 32, 32, noisy.u, noisy.v, None, psize, 1.0)
    chi2 = float(np.sum(np.abs((m - noisy.vis) / noisy.sigma) ** 2))
    print("reduced chi^2 of the noisy observation:", chi2 / (8 * len(noisy)))
    assert 0.85 < chi2 / (8 * len(noisy)) < 1.15


def test_stokes_fits_round_trip_and_movie(tmp_path):
    rng = np.random.default_rng(3)
    img = np.abs(rng.standard_normal((12, 10, 4))) * 1e-3
    M, Dpc, psize_M = 6.5e9, 16.8e6, 0.7
    paths = []
    for k, (mjd, nu) in enumerate([(57854.0, 230e9), (57854.5, 230e9), (57854.0, 345e9), (57854.5, 345e9)]):
        p = tmp_path / f"f{k}.fits"
        fitsio.write_stokes_fits(str(p), img * (1 + k), psize_M, M, Dpc, nu, mjd)
        paths.append(str(p))
    back, hdr = fitsio.read_stokes_fits(paths[0])
    L = fitsio.gravitational_radius(M)
    psize_rad = psize_M * L / (Dpc * fitsio.PC)
    assert hdr["bunit"] == "JY/PIXEL" and hdr["freq"] == 230e9 and hdr["mjd"] == 57854.0
    assert abs(hdr["psize_deg"] * np.pi / 180 - psize_rad) < 1e-12 * psize_rad
    assert np.allclose(back, img * psize_rad ** 2 / 1e-23, rtol=1e-14)
    mv = fitsio.read_stokes_movie(paths[::-1], M, Dpc, sigma=[1e-3, 1e-4, 1e-4, 1e-5])
    assert mv["data"].shape == (12, 10, 2, 2, 4) and list(mv["nus"]) == [230e9, 345e9]
    assert np.allclose(mv["data"][:, :, 1, 1], img * 4, rtol=1e-12)
    assert abs(mv["times"][1] - 0.5 * 86400 / fitsio.time_unit(M)) < 1e-9
    assert mv["camera"].npix == 120 and abs(mv["camera"].alpha[1] - mv["camera"].alpha[0] - psize_M) < 1e-12
