"""Minimal FITS primary-image reader/writer (numpy), written from the FITS standard (4.0):
2880-byte blocks, 80-character header cards, big-endian data. Enough for the imager's
contract: the archive CLI reads 1-D or 2-D images as float (archive/pipe_interface.cpp:12-96,
which uses cfitsio with TFLOAT conversion) and both CLIs write a 2-D FLOAT_IMG
(SVDIntegratedImager.cu:153-176, archive/pipe_interface.cpp:98-137)."""
from __future__ import annotations

import math

import numpy as np

BLOCK = 2880
_BITPIX = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


def _card(key, value, comment=""):
    if isinstance(value, bool):
        v = ("T" if value else "F").rjust(20)
    elif isinstance(value, (int, np.integer)):
        v = str(int(value)).rjust(20)
    elif isinstance(value, float):
        v = f"{value:.15E}".rjust(20)
    else:
        v = ("'" + str(value).replace("'", "''").ljust(8) + "'").ljust(20)
    s = f"{key:<8}= {v}"
    if comment:
        s += " / " + comment
    return s[:80].ljust(80)


def write_fits(path: str, data: np.ndarray, extra_cards=None):
    """Write a primary image; float64 stays BITPIX -64, everything else becomes -32.
    Overwrites an existing file (the reference prefixes the name with '!')."""
    a = np.asarray(data)
    if a.dtype == np.float64:
        bitpix, arr = -64, a.astype(">f8")
    else:
        bitpix, arr = -32, a.astype(">f4")
    cards = [_card("SIMPLE", True, "conforms to FITS standard"), _card("BITPIX", bitpix),
             _card("NAXIS", a.ndim)]
    for i, n in enumerate(a.shape[::-1]):
        cards.append(_card(f"NAXIS{i + 1}", n))
    for k, v in (extra_cards or []):
        cards.append(_card(k, v))
    cards.append("END".ljust(80))
    head = "".join(cards).encode("ascii")
    head += b" " * (-len(head) % BLOCK)
    body = np.ascontiguousarray(arr).tobytes()
    body += b"\0" * (-len(body) % BLOCK)
    with open(path, "wb") as f:
        f.write(head + body)


def sin_wcs_cards(image_size: int, cell_rad: float, ra_deg: float, dec_deg: float):
    """World-coordinate cards of an N x N SIN-projected dirty image (FITS WCS paper II), for
    write_fits(extra_cards=...): reference pixel at the image centre (0-based N // 2, the imager's
    phase centre), cell_rad per pixel, RA decreasing along axis 1 as the imager lays the image
    out, phase centre (ra_deg, dec_deg). The CLIs add the same cards when SVDI_FITS_WCS is set."""
    cell_deg = math.degrees(cell_rad)
    crpix = float(image_size // 2 + 1)
    return [("CTYPE1", "RA---SIN"), ("CRVAL1", float(ra_deg)), ("CRPIX1", crpix), ("CDELT1", -cell_deg),
            ("CUNIT1", "deg"), ("CTYPE2", "DEC--SIN"), ("CRVAL2", float(dec_deg)), ("CRPIX2", crpix),
            ("CDELT2", cell_deg), ("CUNIT2", "deg"), ("RADESYS", "ICRS"), ("EQUINOX", 2000.0),
            ("BUNIT", "JY/BEAM")]


def read_header(raw: bytes):
    hdr, pos = {}, 0
    while True:
        if pos + BLOCK > len(raw):
            raise ValueError("truncated FITS header")
        blk = raw[pos:pos + BLOCK].decode("ascii", errors="replace")
        pos += BLOCK
        for i in range(0, BLOCK, 80):
            c = blk[i:i + 80]
            key = c[:8].strip()
            if key == "END":
                return hdr, pos
            if c[8:10] == "= ":
                raw_val = c[10:].strip()
                if raw_val.startswith("'"):  # quoted string ('' is a quote); a comment may follow
                    j, out = 1, []
                    while j < len(raw_val):
                        if raw_val[j] == "'":
                            if j + 1 < len(raw_val) and raw_val[j + 1] == "'":
                                out.append("'")
                                j += 2
                                continue
                            break
                        out.append(raw_val[j])
                        j += 1
                    hdr[key] = "".join(out).rstrip()
                    continue
                val = raw_val.split("/")[0].strip()
                if val in ("T", "F"):
                    val = val == "T"
                else:
                    try:
                        val = int(val)
                    except ValueError:
                        val = float(val.replace("D", "E"))
                hdr[key] = val


def read_fits(path: str, dtype=np.float32) -> np.ndarray:
    """Read the primary image converted to ``dtype`` (BSCALE/BZERO applied)."""
    with open(path, "rb") as f:
        raw = f.read()
    hdr, pos = read_header(raw)
    naxis = int(hdr.get("NAXIS", 0))
    shape = tuple(int(hdr[f"NAXIS{i}"]) for i in range(naxis, 0, -1))
    n = int(np.prod(shape)) if shape else 0
    bitpix = int(hdr["BITPIX"])
    dt = np.dtype(_BITPIX[bitpix])
    a = np.frombuffer(raw, dtype=dt, count=n, offset=pos).astype(np.float64)
    a = a * float(hdr.get("BSCALE", 1.0)) + float(hdr.get("BZERO", 0.0))
    return a.reshape(shape).astype(dtype)
