"""Generate rr_igm_table.h: the Inoue et al. (2014) Lyman-series tables.

The 39-line table (line wavelength, A_LAF1..3, A_DLA1..2) is the one
published in Inoue, Shimizu, Iwata & Tanaka (2014), Table 2, and shipped by
redrock as py/redrock/data/LAFcoeff.txt and DLAcoeff.txt.  The derived
per-line coefficients A / lambda**gamma are evaluated here with numpy, in the
same expression form as redrock's igm.Inoue14 (igm.py:128-160), and written
as exact hexadecimal floating-point literals so the kernel starts from the
same doubles.

Usage (needs the reference checkout):
    python gen_igm_table.py /path/to/redrock/py/redrock/data > rr_igm_table.h
"""
import os
import sys
import numpy as np


def main(datadir):
    laf = np.loadtxt(f"{datadir}/LAFcoeff.txt", unpack=True)
    dla = np.loadtxt(f"{datadir}/DLAcoeff.txt", unpack=True)
    _, lam, a1, a2, a3 = laf
    _, lam2, d1, d2 = dla
    assert np.array_equal(lam, lam2)
    c_laf = np.stack([a1 / lam ** 1.2, a2 / lam ** 3.7, a3 / lam ** 5.5], axis=1)
    c_dla = np.stack([d1 / lam ** 2, d2 / lam ** 3], axis=1)
    n = len(lam)
    out = []
    out.append("// Generated by gen_igm_table.py -- do not edit.")
    out.append("// Inoue et al. (2014) Lyman-series coefficients (Table 2), one row per line,")
    out.append("// and the derived per-line factors A/lambda^gamma used by the LAF and DLA terms.")
    out.append("#pragma once")
    out.append(f"#define RR_INOUE14_NLINES {n}")
    out.append("static const double rr_inoue14_lam_h[RR_INOUE14_NLINES] = {")
    out += [f"  {float(v).hex()},  // {float(v)!r}" for v in lam]
    out.append("};")
    out.append("// columns: A_LAF1/lam^1.2, A_LAF2/lam^3.7, A_LAF3/lam^5.5")
    out.append("static const double rr_inoue14_laf_h[RR_INOUE14_NLINES][3] = {")
    out += ["  {" + ", ".join(float(v).hex() for v in row) + "}," for row in c_laf]
    out.append("};")
    out.append("// columns: A_DLA1/lam^2, A_DLA2/lam^3")
    out.append("static const double rr_inoue14_dla_h[RR_INOUE14_NLINES][2] = {")
    out += ["  {" + ", ".join(float(v).hex() for v in row) + "}," for row in c_dla]
    out.append("};")
    print("\n".join(out))


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REDROCK_DATA")
    if not src:
        sys.exit("usage: gen_igm_table.py <redrock data directory holding LAFcoeff.txt and "
                 "DLAcoeff.txt> (or set REDROCK_DATA)")
    main(src)
