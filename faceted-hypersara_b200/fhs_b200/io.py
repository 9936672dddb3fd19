"""Files either side of the solver: FITS cubes and MATLAB checkpoints.

* ``fitswrite`` / ``fitsread`` -- the model and residual cubes the reference
  writes with MATLAB's ``fitswrite`` (src/fhs/facetHyperSARA.m:1066-1069,
  1165-1170): one primary HDU, NAXIS1 = the first MATLAB dimension (rows),
  IEEE big-endian data, 2880-byte records (FITS standard 4.0).
* ``save_checkpoint`` / ``load_checkpoint`` -- the solver state under the
  field names of the reference's checkpoint files (facetHyperSARA.m:1071-1107:
  xsol, g, v0, v1, v2, proj, weights0, weights1, epsilon, plus any scalars
  given), as a
  MATLAB v5 MAT-file (readable by MATLAB's ``load``; scipy writes no v7.3
  HDF5 files, so each variable stays below 2 GB: v1 is a cell of per-channel
  columns).  Layouts are this library's (``Solver.get_state``): x, g, weights
  follow the reference; v1 is the global SARA coefficient vector per channel
  rather than the reference's per-facet split.

* ``load_channel_data`` -- one channel's data file as extracted by the
  reference's pyxisMs2mat scripts (fields y, u, v, w, nW, nWimag, frequency,
  maxProjBaseline; pyxisMs2mat/ReadMe.md), converted as the reference does
  before building G: u, v in radians (imaging/imaging.m:387,
  lib/operators/util_load_data_gen_measurement_operator.m), whitened data
  y .* nW (.* nWimag) (imaging/imaging.m:454-464).

Host-side file formats only: nothing here touches the GPU.
"""
from __future__ import annotations

import numpy as np

_BLOCK = 2880
_CARD = 80
_DTYPES = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


def _card(key, value=None, comment=None):
    if value is None:
        text = f"{key:<8}"
    else:
        if isinstance(value, bool):
            v = "T" if value else "F"
        elif isinstance(value, (int, np.integer)):
            v = str(int(value))
        elif isinstance(value, (float, np.floating)):
            v = repr(float(value)).upper()
        else:
            v = "'" + str(value).replace("'", "''").ljust(8) + "'"
        text = f"{key:<8}= {v:>20}"
        if comment:
            text += " / " + comment
    if len(text) > _CARD:
        raise ValueError(f"FITS card too long: {text!r}")
    return text.ljust(_CARD).encode("ascii")


def fitswrite(x, path, bitpix=-64, header=None):
    """Writes array ``x`` (MATLAB order: NAXIS1 = x.shape[0]) to a FITS file.
    ``bitpix`` -64 (float64) or -32 (float32); ``header`` extra (key, value) cards."""
    if bitpix not in (-32, -64):
        raise ValueError("bitpix must be -32 or -64")
    a = np.asarray(x)
    if a.ndim == 0 or a.ndim > 999:
        raise ValueError("FITS arrays need 1 to 999 axes")
    cards = [_card("SIMPLE", True, "conforms to FITS standard"), _card("BITPIX", bitpix),
             _card("NAXIS", a.ndim)]
    cards += [_card(f"NAXIS{i + 1}", n) for i, n in enumerate(a.shape)]
    cards.append(_card("EXTEND", True))
    for k, v in (header or []):
        cards.append(_card(k.upper()[:8], v))
    cards.append(_card("END"))
    head = b"".join(cards)
    head += b" " * (-len(head) % _BLOCK)
    data = np.asarray(a, dtype=_DTYPES[bitpix]).reshape(-1, order="F").tobytes()
    data += b"\0" * (-len(data) % _BLOCK)
    with open(path, "wb") as f:
        f.write(head)
        f.write(data)


def _parse_value(raw):
    v = raw.split("/")[0].strip() if not raw.strip().startswith("'") else raw.strip()
    if v.startswith("'"):
        end = v.find("'", 1)
        while end != -1 and v[end:end + 2] == "''":
            end = v.find("'", end + 2)
        return v[1:end].replace("''", "'").rstrip()
    if v in ("T", "F"):
        return v == "T"
    try:
        return int(v)
    except ValueError:
        return float(v.replace("D", "E"))


def fitsread(path, with_header=False):
    """Reads the primary HDU of a FITS file into an array of MATLAB order
    (shape = (NAXIS1, NAXIS2, ...)); BSCALE / BZERO are applied."""
    with open(path, "rb") as f:
        buf = f.read()
    hdr, pos = {}, 0
    while True:
        if pos + _CARD > len(buf):
            raise ValueError("FITS header without END")
        card = buf[pos:pos + _CARD].decode("ascii")
        pos += _CARD
        key = card[:8].strip()
        if key == "END":
            break
        if card[8:10] == "= ":
            hdr[key] = _parse_value(card[10:])
    pos += -pos % _BLOCK
    if not hdr.get("SIMPLE", False):
        raise ValueError("not a FITS primary HDU")
    bitpix = int(hdr["BITPIX"])
    shape = tuple(int(hdr[f"NAXIS{i + 1}"]) for i in range(int(hdr["NAXIS"])))
    n = int(np.prod(shape)) if shape else 0
    a = np.frombuffer(buf, dtype=_DTYPES[bitpix], count=n, offset=pos).astype(
        np.float64 if bitpix < 0 or "BSCALE" in hdr or "BZERO" in hdr else _DTYPES[bitpix][1:])
    if "BSCALE" in hdr or "BZERO" in hdr:
        a = a * float(hdr.get("BSCALE", 1.0)) + float(hdr.get("BZERO", 0.0))
    a = a.reshape(shape, order="F")
    return (a, hdr) if with_header else a


def _cells(nested):
    """Nested lists [l][b] of arrays -> MATLAB cell (object array, column)."""
    out = np.empty((len(nested), 1), dtype=object)
    for l, row in enumerate(nested):
        c = np.empty((len(row), 1), dtype=object)
        for b, v in enumerate(row):
            c[b, 0] = np.asarray(v).reshape(-1, 1)
        out[l, 0] = c
    return out


def _uncells(c):
    return [[np.asarray(c[l, 0][b, 0]).ravel() for b in range(c[l, 0].shape[0])] for l in range(c.shape[0])]


def save_checkpoint(path, state, **scalars):
    """Writes ``state`` (``Solver.get_state()``) and extra scalars/arrays to a
    MATLAB v5 MAT-file under the reference's field names."""
    from scipy.io import savemat
    d = {}
    for k, v in state.items():
        if k in ("v2", "proj", "epsilon"):
            d[k] = _cells(v)
        elif k == "v1":
            # one [s, L] variable would pass the 2 GB of a v5 variable at large
            # sizes: a cell with one [s, 1] column per channel
            a = np.asarray(v)
            c = np.empty((a.shape[1], 1), dtype=object)
            for l in range(a.shape[1]):
                c[l, 0] = a[:, l:l + 1]
            d[k] = c
        else:
            d[k] = np.asarray(v)
    for k, v in scalars.items():
        d[k] = v
    savemat(path, d, format="5", do_compression=False, oned_as="column")


def load_checkpoint(path):
    """Reads a checkpoint written by save_checkpoint back into the layout of
    ``Solver.get_state``."""
    from scipy.io import loadmat
    m = loadmat(path, squeeze_me=False)
    out = {}
    for k, v in m.items():
        if k.startswith("__"):
            continue
        if k in ("v2", "proj"):
            out[k] = _uncells(v)
        elif k == "epsilon":
            out[k] = [[float(b[0]) for b in bl] for bl in _uncells(v)]
        elif k == "v0":
            out[k] = np.asarray(v).ravel(order="F")
        elif k == "v1":
            out[k] = np.concatenate([np.asarray(v[l, 0]).reshape(-1, 1) for l in range(v.shape[0])], axis=1)
        else:
            out[k] = np.asarray(v)
    return out


SPEED_OF_LIGHT = 299792458.0


def half_spatial_bandwidth(pixel_size_arcsec):
    """imaging/imaging.m:387: (180/pi) 3600 / pixelSize / 2."""
    return (180.0 / np.pi) * 3600.0 / float(pixel_size_arcsec) / 2.0


def nominal_pixel_size(max_proj_baseline, superresolution=2.0):
    """imaging/imaging.m:372-385: pixel size (arcsec) when none is given, from
    the largest projected baseline (in wavelengths) of the imaged channels."""
    return (180.0 / np.pi) * 3600.0 / (superresolution * 2.0 * float(max_proj_baseline))


def load_channel_data(path, pixel_size_arcsec, apply_imaging_weights=True):
    """Reads one channel's data file and returns dict(y, om_y, om_x, weights,
    w, frequency, max_proj_baseline) ready for ``MeasurementOperator``
    (om = (v, u) in radians, weights = nW [.* nWimag]) and the solvers
    (y whitened by the same weights)."""
    from scipy.io import loadmat
    m = loadmat(path, squeeze_me=True)
    hsb = half_spatial_bandwidth(pixel_size_arcsec)
    u = np.asarray(m["u"], dtype=np.float64).ravel() * np.pi / hsb
    v = -np.asarray(m["v"], dtype=np.float64).ravel() * np.pi / hsb
    nW = np.asarray(m["nW"], dtype=np.float64).ravel()
    if apply_imaging_weights and "nWimag" in m and np.size(m["nWimag"]) == nW.size:
        nW = nW * np.asarray(m["nWimag"], dtype=np.float64).ravel()
    y = np.asarray(m["y"]).astype(np.complex128).ravel() * nW
    out = dict(y=y, om_y=v, om_x=u, weights=nW,
               w=np.asarray(m["w"], dtype=np.float64).ravel() if "w" in m else None,
               frequency=float(np.asarray(m["frequency"]).ravel()[0]) if "frequency" in m else None,
               max_proj_baseline=float(np.asarray(m["maxProjBaseline"]).ravel()[0])
               if "maxProjBaseline" in m else None)
    return out
