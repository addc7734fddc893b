"""ipole's RIAF on the GPU (ks_riaf_image): the GPU's own frames, field transport and polarized
step against ipole's full-Stokes images under the reference's gate (test/test_polarized.jl:156-178,
the same comparison tests/test_riaf_ipole.py makes for the oracle), and against the oracle on the
same rays: FP64 within 1e-10 relative Stokes L2 (whole sample and per lit pixel), the FP32 transport
(KS_MIXED) within 1e-4."""
import numpy as np
import pytest

import kerrsplat_b200 as ks
from test_riaf_ipole import A, THETA_O, gate, ipole_reference, riaf_camera

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def riaf_run():
    alpha, beta, L, scale = riaf_camera()
    cam = ks.Camera(alpha, beta)
    cache = ks.GeodesicCache(cam, 2000)
    ks.regenerate(cache, A, THETA_O, marcher=ks.Fused(64))
    model = ks.RIAFModel.example(A)
    nus = np.array([230e9, 2e12])
    out64 = ks.riaf_image(cache, model, nus, L, precision=ks.KS_FP64)
    out32 = ks.riaf_image(cache, model, nus, L, precision=ks.KS_MIXED)
    yield dict(alpha=alpha, beta=beta, L=L, scale=scale, nus=nus, out64=out64, out32=out32)
    cache.close()


@pytest.mark.parametrize("f,tag", [(0, "fine"), (1, "2thz")])
@pytest.mark.parametrize("prec", ["out64", "out32"])
def test_gpu_riaf_matches_ipole(riaf_run, f, tag, prec):
    ours = riaf_run[prec][f]
    res, tot, dchi, lp, lpr = gate(ours, ipole_reference(tag), riaf_run["scale"])
    msg = f"{prec} {tag}: residuals {res}, totals {tot}, dchi {dchi:.2e}, lp {lp:.4f} vs {lpr:.4f}"
    print(msg)
    assert np.all(res < 0.03) and np.all(np.abs(tot - 1) < 0.01) and dchi < 0.01 and abs(lp - lpr) < 0.005, msg


def test_gpu_riaf_matches_oracle(riaf_run, oracle):
    r = riaf_run
    sel = np.arange(0, r["alpha"].size, 5)
    oracle.set_threads(max(1, oracle.num_threads()))
    for f, nu in enumerate(r["nus"]):
        ref = oracle.riaf_image(A, THETA_O, r["alpha"][sel], r["beta"][sel], 2000, 64, nu, r["L"])
        got64, got32 = r["out64"][f][sel], r["out32"][f][sel]
        nr = np.linalg.norm(ref, axis=1)
        lit = nr > 1e-6 * nr.max()
        pix = np.linalg.norm(got64 - ref, axis=1)[lit] / nr[lit]
        tot64 = np.linalg.norm(got64 - ref) / np.linalg.norm(ref)
        tot32 = np.linalg.norm(got32 - ref) / np.linalg.norm(ref)
        print(f"RIAF {nu / 1e9:.0f} GHz: FP64 {tot64:.2e} (worst lit pixel {pix.max():.2e}), FP32 transport {tot32:.2e}")
        assert tot64 < 1e-10 and pix.max() < 1e-10
        assert tot32 < 1e-4
