"""Stokes images, movies and uvfits observations: the data formats on either side of the render path
(src/Fit/fits.jl and src/Fit/uvfits.jl), read and written with numpy alone.

The FITS layer handles what these files use: primary and IMAGE HDUs (BITPIX 8/16/32/64/-32/-64 with
BSCALE/BZERO), the random-groups primary HDU of uvfits (GROUPS = T: PCOUNT parameters then the data
array per group, parameters scaled by PSCALn/PZEROn) and BINTABLE extensions of fixed-width columns
(TFORM codes L, B, I, J, K, A, E, D, C, M). Header cards are 80 characters in 2880-byte blocks,
data big-endian, the first axis (NAXIS1) fastest: an image comes back as an (NAXIS1, NAXIS2) array
indexed (x, y), as the reference reads it.
"""
import math
import os

import numpy as np

from . import Camera, JY, gravitational_radius

__all__ = ["read_fits", "read_stokes_fits", "write_stokes_fits", "read_stokes_movie", "read_uvfits", "antenna_positions", "Observation",
           "time_unit", "PC"]

PC = 3.085678e18      # cm (constants.jl)
BLOCK = 2880
_BITPIX = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}
_TFORM = {"L": ("?", 1), "B": (">u1", 1), "I": (">i2", 2), "J": (">i4", 4), "K": (">i8", 8), "E": (">f4", 4), "D": (">f8", 8),
          "C": (">c8", 8), "M": (">c16", 16)}


def time_unit(M_solar):
    """GM/c^3 in seconds for a mass in solar masses (fits.jl:7)."""
    return gravitational_radius(M_solar) / 2.99792458e10


# ---- the FITS layer ----------------------------------------------------------------------------

def _parse_value(s):
    s = s.strip()
    if s.startswith("'"):
        end = s.find("'", 1)
        while end != -1 and end + 1 < len(s) and s[end + 1] == "'":     # '' is a quote inside a string
            end = s.find("'", end + 2)
        return s[1:end].replace("''", "'").rstrip()
    v = s.split("/")[0].strip()
    if v == "T":
        return True
    if v == "F":
        return False
    try:
        return int(v)
    except ValueError:
        pass
    try:
        return float(v.replace("D", "E"))
    except ValueError:
        return v


class HDU:
    """One header-data unit: `header` (ordered keyword -> value), `data` (numpy array, random-groups
    tuple (params, data) or structured table), `kind` ("image", "groups", "table")."""

    def __init__(self, header, data, kind):
        self.header, self.data, self.kind = header, data, kind

    def get(self, key, default=None):
        return self.header.get(key, default)


def _read_header(buf, off):
    header = {}
    while True:
        if off + BLOCK > len(buf):
            raise ValueError("truncated FITS header")
        blk = buf[off:off + BLOCK]
        off += BLOCK
        done = False
        for i in range(0, BLOCK, 80):
            card = blk[i:i + 80].decode("ascii", errors="replace")
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= " and key:
                header[key] = _parse_value(card[10:])
        if done:
            return header, off


def _table(header, raw):
    fields, pos = [], 0
    for k in range(1, int(header["TFIELDS"]) + 1):
        form = str(header[f"TFORM{k}"]).strip()
        i = 0
        while i < len(form) and form[i].isdigit():
            i += 1
        rep = int(form[:i]) if i else 1
        code = form[i]
        name = str(header.get(f"TTYPE{k}", f"COL{k}")).strip()
        if code == "A":
            fields.append((name, f"S{rep}", pos))
            pos += rep
        elif code == "X":
            fields.append((name, f"V{(rep + 7) // 8}", pos))
            pos += (rep + 7) // 8
        else:
            dt, size = _TFORM[code]
            fields.append((name, (dt, (rep,)) if rep != 1 else dt, pos))
            pos += rep * size
    dtype = np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields], "offsets": [f[2] for f in fields],
                      "itemsize": int(header["NAXIS1"])})
    return np.frombuffer(raw, dtype=dtype, count=int(header["NAXIS2"]))


def read_fits(path):
    """Every HDU of a FITS file (see HDU)."""
    with open(path, "rb") as f:
        buf = f.read()
    hdus, off = [], 0
    while off + BLOCK <= len(buf):
        if not buf[off:off + 80].strip(b" \x00"):
            break
        header, off = _read_header(buf, off)
        bitpix = int(header.get("BITPIX", 8))
        naxis = int(header.get("NAXIS", 0))
        dims = [int(header.get(f"NAXIS{i}", 0)) for i in range(1, naxis + 1)]
        pcount, gcount = int(header.get("PCOUNT", 0)), int(header.get("GCOUNT", 1))
        item = abs(bitpix) // 8
        if header.get("GROUPS") is True and naxis > 0 and dims[0] == 0:
            per = math.prod(dims[1:])
            nbytes = item * gcount * (pcount + per)
            raw = np.frombuffer(buf, dtype=_BITPIX[bitpix], count=gcount * (pcount + per), offset=off).astype(np.float64)
            raw = raw.reshape(gcount, pcount + per)
            data, kind = (raw[:, :pcount], raw[:, pcount:]), "groups"
        elif str(header.get("XTENSION", "")).strip() == "BINTABLE":
            nbytes = dims[0] * dims[1] + pcount
            data, kind = _table(header, buf[off:off + dims[0] * dims[1]]), "table"
        else:
            n = math.prod(dims) if naxis else 0
            nbytes = item * n * (gcount if "XTENSION" in header else 1) + (item * pcount if "XTENSION" in header else 0)
            arr = np.frombuffer(buf, dtype=_BITPIX[bitpix], count=n, offset=off).astype(np.float64) if n else np.zeros(0)
            arr = arr * float(header.get("BSCALE", 1.0)) + float(header.get("BZERO", 0.0))
            data, kind = (arr.reshape(dims[::-1]).T if n else arr), "image"
        hdus.append(HDU(header, data, kind))
        off += (nbytes + BLOCK - 1) // BLOCK * BLOCK
    return hdus


def _card(key, value, comment=""):
    if isinstance(value, bool):
        v = f"{'T' if value else 'F':>20}"
    elif isinstance(value, (int, np.integer)):
        v = f"{int(value):>20}"
    elif isinstance(value, (float, np.floating)):
        s = repr(float(value)).upper()
        if "E" not in s and "." not in s:
            s += ".0"
        v = f"{s:>20}"
    else:
        s = str(value).replace("'", "''")
        v = f"'{s:<8}'"
    card = f"{key:<8}= {v}" + (f" / {comment}" if comment else "")
    if len(card) > 80:
        raise ValueError(f"FITS card too long: {card}")
    return card.ljust(80)


def _write_hdu(f, cards, data):
    text = "".join(cards) + "END".ljust(80)
    text += " " * ((-len(text)) % BLOCK)
    f.write(text.encode("ascii"))
    raw = np.ascontiguousarray(data.T, dtype=">f8").tobytes()   # NAXIS1 (x) fastest
    f.write(raw + b"\x00" * ((-len(raw)) % BLOCK))


# ---- Stokes images and movies (fits.jl) ---------------------------------------------------------

def read_stokes_fits(path):
    """An ehtim-style FITS image (read_stokes_fits, fits.jl:19-44): the HDUs with STOKES = I, Q, U, V
    (a missing one counts as zero; the first image HDU without the keyword is I) as an (nx, ny, 4)
    array in the file's units, and the header quantities psize_deg (|CDELT2|), freq (Hz), mjd, bunit."""
    imgs, hdr = {}, None
    for h in read_fits(path):
        if h.kind != "image" or h.data.ndim != 2:
            continue
        if hdr is None:
            hdr = h.header
        st = str(h.get("STOKES", "I" if not imgs else " ")).strip().upper()[:1]
        if st in "IQUV" and st:
            imgs[st] = h.data
    if "I" not in imgs:
        raise ValueError(f"no Stokes I image in {path}")
    n = imgs["I"].shape
    S = np.stack([imgs.get(c, np.zeros(n)) for c in "IQUV"], axis=-1)
    header = dict(psize_deg=abs(float(hdr.get("CDELT2", hdr.get("CDELT1")))), freq=float(hdr.get("FREQ", float("nan"))),
                  mjd=float(hdr.get("MJD", float("nan"))), bunit=str(hdr.get("BUNIT", "JY/PIXEL")).strip().upper())
    return S, header


def write_stokes_fits(path, image, psize_M, M_solar, D_pc, freq, mjd, source="KerrSplat"):
    """An (nx, ny, 4) Stokes image in cgs intensity (x toward west = +alpha, y toward north) as an
    ehtim-style FITS file in Jy/pixel, one HDU per Stokes parameter (write_stokes_fits,
    fits.jl:55-104)."""
    L = gravitational_radius(M_solar)
    D = D_pc * PC
    psize_rad = psize_M * L / D
    omega = psize_rad ** 2
    image = np.asarray(image, dtype=np.float64)
    nx, ny = image.shape[:2]
    deg = psize_rad * 180 / math.pi
    with open(path, "wb") as f:
        for k, st in enumerate("IQUV"):
            head = [_card("SIMPLE", True), _card("BITPIX", -64), _card("NAXIS", 2), _card("NAXIS1", nx), _card("NAXIS2", ny),
                    _card("EXTEND", True)] if k == 0 else \
                   [_card("XTENSION", "IMAGE"), _card("BITPIX", -64), _card("NAXIS", 2), _card("NAXIS1", nx), _card("NAXIS2", ny),
                    _card("PCOUNT", 0), _card("GCOUNT", 1)]
            head += [_card("OBJECT", source), _card("CTYPE1", "RA---SIN"), _card("CTYPE2", "DEC--SIN"), _card("CDELT1", -deg),
                     _card("CDELT2", deg), _card("CRPIX1", (nx + 1) / 2), _card("CRPIX2", (ny + 1) / 2), _card("CRVAL1", 0.0),
                     _card("CRVAL2", 0.0), _card("CUNIT1", "deg"), _card("CUNIT2", "deg"), _card("FREQ", float(freq)),
                     _card("MJD", float(mjd)), _card("BUNIT", "JY/PIXEL"), _card("STOKES", st), _card("TELESCOP", "KerrSplat")]
            _write_hdu(f, head, image[:, :, k] * omega / JY)
    return path


def read_stokes_movie(paths, M_solar, D_pc, sigma, mjd0=None, freq=None):
    """A Stokes movie from ehtim-style FITS images, one file per (time, frequency) (read_stokes_movie,
    fits.jl:46-88): intensities to cgs by the pixel solid angle, times to M from mjd0 (default the
    earliest frame), the pixel grid as a Camera in M. Returns dict(data (nx, ny, ntimes, nfreqs, 4),
    times, nus, sigma (4, cgs), camera, L)."""
    L = gravitational_radius(M_solar)
    D = D_pc * PC
    frames = [read_stokes_fits(p) + (p,) for p in paths]
    h1 = frames[0][1]
    psize_rad = h1["psize_deg"] * math.pi / 180
    nx, ny = frames[0][0].shape[:2]
    if h1["bunit"] != "JY/PIXEL":
        raise ValueError(f"unsupported BUNIT {h1['bunit']}")
    tojy = JY / psize_rad ** 2
    mjds = [fr[1]["mjd"] for fr in frames]
    freqs = []
    for fr in frames:
        if math.isnan(fr[1]["freq"]):
            if freq is None:
                raise ValueError(f"no FREQ in {fr[2]}")
            freqs.append(float(freq))
        else:
            freqs.append(fr[1]["freq"])
    t0 = min(mjds) if mjd0 is None else mjd0
    times, nus = sorted(set(mjds)), sorted(set(freqs))
    data = np.zeros((nx, ny, len(times), len(nus), 4))
    filled = np.zeros((len(times), len(nus)), dtype=bool)
    for fr, mjd, nu in zip(frames, mjds, freqs):
        if fr[0].shape[:2] != (nx, ny):
            raise ValueError("image sizes differ across the movie")
        k, l = times.index(mjd), nus.index(nu)
        data[:, :, k, l] = fr[0] * tojy
        filled[k, l] = True
    if not filled.all():
        raise ValueError("the movie does not cover every (time, frequency) pair")
    tM = (np.array(times) - t0) * 86400 / time_unit(M_solar)
    psize_M = psize_rad * D / L
    ax = (np.arange(1, nx + 1) - (nx + 1) / 2) * psize_M
    ay = (np.arange(1, ny + 1) - (ny + 1) / 2) * psize_M
    cam = Camera(np.tile(ax, ny), np.repeat(ay, nx))
    cam.size = (nx, ny)
    return dict(data=data, times=tM, nus=np.array(nus), sigma=np.asarray(sigma, dtype=np.float64) * tojy, camera=cam, L=L)


# ---- uvfits (uvfits.jl) -------------------------------------------------------------------------

class Observation:
    """Visibilities of a uvfits file (Observation, uvfits.jl:9-35): per row time (UT hours of day
    mjd), tint (s), station indices s1, s2 into `stations`, baseline u, v (wavelengths), Stokes
    visibilities vis (n, 4) complex Jy and noise sigma (n, 4) Jy (inf for a missing parameter); the
    circular products coh (RR, LL, RL, LR) with sigma_coh; freq, bandwidth (Hz), ra (h), dec (deg),
    mjd, source."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def __len__(self):
        return len(self.u)


def _products_from_stokes(vis, sig):
    sP = math.sqrt(sig[0] ** 2 + sig[3] ** 2)
    sX = math.sqrt(sig[1] ** 2 + sig[2] ** 2)
    return [vis[0] + vis[3], vis[0] - vis[3], vis[1] + 1j * vis[2], vis[1] - 1j * vis[2]], [sP, sP, sX, sX]


def read_uvfits(path):
    """A random-groups uvfits file (read_uvfits, uvfits.jl:91-205): UU, VV scaled to wavelengths by
    the antenna table's reference frequency, baselines decoded as 256 a1 + a2, the two DATE
    parameters summed to a Julian date, the correlation products averaged over channels and IFs
    where their weights are positive and finite (noise sqrt(sum 1/w) / n), and converted to Stokes
    (I = (RR + LL)/2, Q = (RL + LR)/2, U = (RL - LR)/(2i), V = (RR - LL)/2, noise in quadrature).
    Rows without parallel hands are dropped; one parallel hand alone is I without V; missing cross
    hands leave Q and U with infinite noise."""
    hdus = read_fits(path)
    prim = hdus[0]
    h = prim.header
    if prim.kind != "groups":
        raise ValueError(f"{path} is not a random-groups uvfits file")
    npar = int(h["PCOUNT"])
    naxis = int(h["NAXIS"])
    dims = [int(h[f"NAXIS{i}"]) for i in range(2, naxis + 1)]
    ctypes = [str(h.get(f"CTYPE{i}", "")).strip().upper() for i in range(2, naxis + 1)]
    ptypes = [str(h[f"PTYPE{i}"]).strip().upper() for i in range(1, npar + 1)]
    pscal = np.array([float(h.get(f"PSCAL{i}", 1.0)) for i in range(1, npar + 1)])
    pzero = np.array([float(h.get(f"PZERO{i}", 0.0)) for i in range(1, npar + 1)])
    if not (ctypes[0] == "COMPLEX" and ctypes[1] == "STOKES" and "FREQ" in ctypes):
        raise ValueError(f"unsupported axis order {ctypes} in {path}")
    if dims[0] != 3:
        raise ValueError(f"expected (re, im, weight) triples on the COMPLEX axis of {path}")
    ifreq = ctypes.index("FREQ")
    iif = ctypes.index("IF") if "IF" in ctypes else None
    nstokes, nchan = dims[1], dims[ifreq]
    nif = dims[iif] if iif is not None else 1
    stokes0 = int(round(float(h["CRVAL3"])))
    dst = int(round(float(h.get("CDELT3", 1.0))))
    codes = [stokes0 + k * dst for k in range(nstokes)]       # -1..-4 = RR, LL, RL, LR; 1..4 = I, Q, U, V
    circular = all(c < 0 for c in codes)
    if not circular and not all(c > 0 for c in codes):
        raise ValueError(f"mixed STOKES axis {codes} in {path}")
    slot = lambda code: codes.index(code) if code in codes else None
    ra = float(h.get(f"CRVAL{ifreq + 4}", float("nan"))) * 12 / 180
    dec = float(h.get(f"CRVAL{ifreq + 5}", float("nan")))
    for i in range(2, naxis + 1):
        if ctypes[i - 2] == "RA":
            ra = float(h[f"CRVAL{i}"]) * 12 / 180
        if ctypes[i - 2] == "DEC":
            dec = float(h[f"CRVAL{i}"])
    source = str(h.get("OBJECT", "")).strip()
    ch1 = float(h[f"CRVAL{ifreq + 2}"])
    bandwidth = abs(float(h.get(f"CDELT{ifreq + 2}", float("nan"))))
    stations, nosta, rf = [], [], ch1
    for t in hdus[1:]:
        if t.kind == "table" and str(t.get("EXTNAME", "")).strip().upper() == "AIPS AN":
            stations = [s.decode("ascii").strip() for s in t.data["ANNAME"]]
            nosta = [int(x) for x in t.data["NOSTA"]]
            if "FREQ" in t.header:
                rf = float(t.header["FREQ"])
    if not stations:
        raise ValueError(f"no AIPS AN table in {path}")
    order = np.argsort(nosta, kind="stable")
    stations = [stations[i] for i in order]
    nosta = [nosta[i] for i in order]

    def station_index(n):
        if n not in nosta:
            raise ValueError(f"baseline refers to station {n} absent from the AN table")
        return nosta.index(n)

    find = lambda pred: next((i for i, p in enumerate(ptypes) if pred(p)), None)
    iu, iv = find(lambda p: p.startswith("UU")), find(lambda p: p.startswith("VV"))
    ibl, itint = find(lambda p: p == "BASELINE"), find(lambda p: p == "INTTIM")
    idates = [i for i, p in enumerate(ptypes) if p == "DATE"]
    if iu is None or iv is None or ibl is None or not idates:
        raise ValueError(f"missing UU/VV/BASELINE/DATE parameters in {path}")
    pars_all, block_all = prim.data
    # the data of a group: (re, im, weight) fastest, then STOKES, then FREQ, IF, ...
    stride_chan = 3 * nstokes
    stride_if = 3 * nstokes * math.prod(dims[2:iif]) if iif is not None else 0
    out = {k: [] for k in ("time", "tint", "s1", "s2", "u", "v", "vis", "sigma", "jd", "coh", "sigma_coh")}
    for g in range(pars_all.shape[0]):
        pars, block = pars_all[g], block_all[g]
        mean = np.full(nstokes, np.nan + 0j)
        sig = np.full(nstokes, np.inf)
        for p in range(nstokes):
            acc, var, n = 0j, 0.0, 0
            for m in range(nif):
                for c in range(nchan):
                    base = 3 * p + stride_chan * c + stride_if * m
                    w = block[base + 2]
                    if not (np.isfinite(w) and w > 0):
                        continue
                    acc += complex(block[base], block[base + 1])
                    var += 1 / w
                    n += 1
            if n:
                mean[p] = acc / n
                sig[p] = math.sqrt(var) / n
        jd = float(sum(pscal[i] * pars[i] + pzero[i] for i in idates))
        if circular:
            rr, ll, rl, lr = slot(-1), slot(-2), slot(-3), slot(-4)
            hasrr = rr is not None and np.isfinite(sig[rr])
            hasll = ll is not None and np.isfinite(sig[ll])
            if not (hasrr or hasll):
                continue
            if hasrr and hasll:
                I, V = (mean[rr] + mean[ll]) / 2, (mean[rr] - mean[ll]) / 2
                sI = math.sqrt(sig[rr] ** 2 + sig[ll] ** 2) / 2
                sV = sI
            else:
                I, V = (mean[rr], 0j) if hasrr else (mean[ll], 0j)
                sI, sV = (sig[rr] if hasrr else sig[ll]), math.inf
            cross = rl is not None and lr is not None and np.isfinite(sig[rl]) and np.isfinite(sig[lr])
            Q = (mean[rl] + mean[lr]) / 2 if cross else 0j
            U = (mean[rl] - mean[lr]) / 2j if cross else 0j
            sQ = math.sqrt(sig[rl] ** 2 + sig[lr] ** 2) / 2 if cross else math.inf
            out["vis"].append([I, Q, U, V])
            out["sigma"].append([sI, sQ, sQ, sV])
            prod = lambda j: (0j, math.inf) if j is None or not np.isfinite(sig[j]) else (mean[j], sig[j])
            pr = [prod(j) for j in (rr, ll, rl, lr)]
            out["coh"].append([x[0] for x in pr])
            out["sigma_coh"].append([x[1] for x in pr])
        else:
            si = slot(1)
            if si is None or not np.isfinite(sig[si]):
                continue
            comp = lambda k: (0j, math.inf) if slot(k) is None or not np.isfinite(sig[slot(k)]) else (mean[slot(k)], sig[slot(k)])
            (Q, sQ), (U, sU), (V, sV) = comp(2), comp(3), comp(4)
            out["vis"].append([mean[si], Q, U, V])
            out["sigma"].append([sig[si], sQ, sU, sV])
            c_, s_ = _products_from_stokes(out["vis"][-1], out["sigma"][-1])
            out["coh"].append(c_)
            out["sigma_coh"].append(s_)
        bl = int(math.floor(pscal[ibl] * pars[ibl] + pzero[ibl]))
        a1, a2 = bl // 256, bl - 256 * (bl // 256)
        out["s1"].append(station_index(a1))
        out["s2"].append(station_index(a2))
        out["u"].append((pscal[iu] * pars[iu] + pzero[iu]) * rf)
        out["v"].append((pscal[iv] * pars[iv] + pzero[iv]) * rf)
        out["jd"].append(jd)
        out["tint"].append(pscal[itint] * pars[itint] + pzero[itint] if itint is not None else 0.0)
    if not out["jd"]:
        raise ValueError(f"no unflagged parallel-hand data in {path}")
    jds = np.array(out["jd"])
    mjd = int(math.floor(jds.min() - 2400000.5))
    return Observation(time=(jds - 2400000.5 - mjd) * 24, tint=np.array(out["tint"]), s1=np.array(out["s1"]), s2=np.array(out["s2"]),
                       stations=stations, u=np.array(out["u"]), v=np.array(out["v"]), vis=np.array(out["vis"], dtype=np.complex128),
                       sigma=np.array(out["sigma"]), freq=rf, bandwidth=bandwidth, ra=ra, dec=dec, mjd=mjd, source=source,
                       coh=np.array(out["coh"], dtype=np.complex128), sigma_coh=np.array(out["sigma_coh"]))


def antenna_positions(path):
    """Geocentric station positions (m) from the STABXYZ column of the AIPS AN table, by name
    (antenna_positions, uvfits.jl:236-251)."""
    for t in read_fits(path)[1:]:
        if t.kind == "table" and str(t.get("EXTNAME", "")).strip().upper() == "AIPS AN":
            return {s.decode("ascii").strip(): np.array(xyz, dtype=np.float64) for s, xyz in zip(t.data["ANNAME"], t.data["STABXYZ"])}
    raise ValueError(f"no AIPS AN table in {path}")
