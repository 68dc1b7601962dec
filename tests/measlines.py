"""Measurements as the reference prints them (control.c:52-68, 85-138).

Builds, from a measurement dict (susy_b200.Lattice.measure() or the
oracle's measurements()), the numbers of each output line, and compares
them with the reference's printed lines to the precision they were printed
with (%.6g or %.8g: a relative tolerance of a few units in the last printed
digit).
"""
import numpy as np

# significant digits each line is printed with
DIGITS = {"FLINK": 6, "FLINK_DET": 6, "GMES": 8, "BACTION": 8, "LINES": 6,
          "LINES_POLAR": 6, "DET": 6, "WIDTHS": 6, "UUBAR_EIG": 6, "POLAR_EIG": 6}


def printed(m, volume, iters=0):
    """tag -> list of numbers, as the reference would print them"""
    inter = lambda z: [v for c in z for v in (c.real, c.imag)]
    out = {
        "FLINK": list(m["linktr"]) + [m["linktr_ave"], m["linktr_width"]],
        "FLINK_DET": list(m["link_det"]) + [m["det_ave"], m["det_width"]],
        "GMES": [m["ploop_re"], m["ploop_im"], iters, m["ss_plaq"], m["st_plaq"],
                 m["gauge_action"] / volume, m["ploop_mod"]],
        "BACTION": [m["gauge_action"] / volume],
        "LINES": inter(m["lines"]),
        "LINES_POLAR": inter(m["lines_polar"]),
        "DET": list(m["det"]),
        "WIDTHS": list(m["widths"]),
        "UUBAR_EIG": [list(x) for x in np.array(m["uubar"]).T],
        "POLAR_EIG": [list(x) for x in np.array(m["polar"]).T],
    }
    return out


def mismatches(got, want_lines, skip=()):
    """[(tag, index, got, want)] for numbers outside printed precision"""
    bad = []
    for tag, want in want_lines.items():
        if tag in skip:
            continue
        g = np.array(got[tag], dtype=float).ravel()
        w = np.array(want, dtype=float).ravel()
        tol = 3.0 * 10.0 ** (1 - DIGITS[tag])
        for k, (a, b) in enumerate(zip(g, w)):
            if abs(a - b) > tol * abs(b) + 1e-12:
                bad.append((tag, k, a, b))
    return bad
