"""Generate tests/golden/{cheb,mode}_U{2,3}.json from the reference's own files.

The reference's measurement programs susy_cheb (Chebyshev coefficients of
the spectral density, 4d_Q16/susy/chebyshev.c, which applies DSq) and
susy_mode (the stochastic mode number, modenumber.c, which calls
congrad_multi) have regression runs testsuite/in.U<N>.{cheb,mode} with
outputs testsuite/scalar/{cheb,mode}.U<N>.ref.  This keeps, per program and
NCOL, the run's input as ordered (key, value) pairs and the printed result
lines: CHEBYSHEV c[k] value error, and the Step function line plus MODE
omega value error.

Run where the reference sources exist:

    python tests/golden/make_golden_apps.py
"""
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SUSY_REFERENCE", "/root/reference") + "/4d_Q16/testsuite"


def parse_input(path):
    pairs = []
    for line in open(path):
        p = line.split()
        if len(p) == 2:
            pairs.append(p)
        elif len(p) == 1 and p[0] in ("forget", "fresh"):
            pass
    return pairs


def parse_output(txt):
    out = {"chebyshev": [], "mode": [], "step": None}
    for m in re.finditer(r"^CHEBYSHEV c\[(\d+)\] (\S+) (\S+)$", txt, re.M):
        out["chebyshev"].append([int(m.group(1)), float(m.group(2)), float(m.group(3))])
    for m in re.finditer(r"^MODE (\S+) (\S+) (\S+)$", txt, re.M):
        out["mode"].append([float(m.group(1)), float(m.group(2)), float(m.group(3))])
    m = re.search(r"^Step function order (\d+) epsilon (\S+) delta (\S+) star (\S+)$", txt, re.M)
    if m:
        out["step"] = [float(x) for x in m.groups()]
    return out


def main():
    for prog in ("cheb", "mode"):
        for N in (2, 3):
            d = {"input": parse_input(os.path.join(REF, "in.U%d.%s" % (N, prog)))}
            d.update(parse_output(open(os.path.join(REF, "scalar/%s.U%d.ref" % (prog, N))).read()))
            path = os.path.join(HERE, "%s_U%d.json" % (prog, N))
            with open(path, "w") as f:
                json.dump(d, f, indent=1)
            print(path, len(d["chebyshev"]), len(d["mode"]))


if __name__ == "__main__":
    main()
