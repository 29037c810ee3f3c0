"""A minimal reader of FITS binary tables (the redrock archetype files,
rrarchetype-*.fits: an ARCHETYPES table with ARCHETYPE and SUBTYPE columns
and the wavelength grid in CRVAL1 / CDELT1 / LOGLAM), for when astropy is
not installed.  Follows the FITS standard 4.0: 2880-byte blocks of 80-char
header cards; BINTABLE rows of big-endian fields (TFORMn: rL, rB, rI, rJ,
rK, rE, rD, rA)."""

from __future__ import annotations

import os

import numpy as np

_BLOCK = 2880
_TFORM = {"L": "b1", "B": "u1", "I": ">i2", "J": ">i4", "K": ">i8", "E": ">f4", "D": ">f8"}


def _value(v):
    v = v.split("/")[0].strip() if not v.strip().startswith("'") else v.strip()
    if v.startswith("'"):
        end = v.find("'", 1)
        while end != -1 and end + 1 < len(v) and v[end + 1] == "'":
            end = v.find("'", end + 2)
        return v[1:end].replace("''", "'").rstrip()
    if v in ("T", "F"):
        return v == "T"
    try:
        return int(v)
    except ValueError:
        try:
            return float(v.replace("D", "E"))
        except ValueError:
            return v


class HDU:
    def __init__(self, header, data):
        self.header = header
        self.data = data


def read_hdus(filename):
    """[HDU] of a FITS file: header dicts and, for BINTABLE extensions, the
    rows as a numpy structured array (native byte order)."""
    with open(os.path.expandvars(filename), "rb") as f:
        raw = f.read()
    out = []
    off = 0
    while off < len(raw):
        header = {}
        done = False
        while not done:
            block = raw[off:off + _BLOCK]
            if len(block) < _BLOCK:
                raise ValueError("truncated FITS header")
            off += _BLOCK
            for i in range(36):
                card = block[80 * i:80 * (i + 1)].decode("ascii")
                key = card[:8].strip()
                if key == "END":
                    done = True
                    break
                if card[8:10] == "= ":
                    header[key] = _value(card[10:])
        naxis = header.get("NAXIS", 0)
        nbytes = 0
        if naxis:
            nbytes = abs(header["BITPIX"]) // 8
            for k in range(1, naxis + 1):
                nbytes *= header[f"NAXIS{k}"]
            nbytes += header.get("PCOUNT", 0)
        data = None
        if header.get("XTENSION") == "BINTABLE":
            fields = []
            for k in range(1, header["TFIELDS"] + 1):
                form = header[f"TFORM{k}"].strip()
                rep = int(form[:-1]) if len(form) > 1 else 1
                code = form[-1]
                name = header.get(f"TTYPE{k}", f"col{k}").strip()
                if code == "A":
                    fields.append((name, f"S{rep}"))
                elif code in _TFORM:
                    fields.append((name, _TFORM[code], (rep,)) if rep != 1 else
                                  (name, _TFORM[code]))
                else:
                    raise ValueError(f"TFORM {form!r} is not supported")
            dt = np.dtype(fields)
            if dt.itemsize != header["NAXIS1"]:
                raise ValueError("row size does not match NAXIS1")
            rows = np.frombuffer(raw, dtype=dt, count=header["NAXIS2"], offset=off)
            data = rows.astype(dt.newbyteorder("=")) if dt.byteorder != "=" else rows.copy()
            data = data.astype([(n, dt.fields[n][0].newbyteorder("="))
                                for n in dt.names])
        out.append(HDU(header, data))
        off += -(-nbytes // _BLOCK) * _BLOCK
    return out


def read_table(filename, extname):
    """(header, rows) of the BINTABLE extension named extname."""
    for h in read_hdus(filename):
        if h.header.get("EXTNAME", "").strip() == extname:
            return h.header, h.data
    raise KeyError(extname)
