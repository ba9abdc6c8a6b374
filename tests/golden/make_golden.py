"""Generate the golden fixtures that pin the oracle to the reference's own tests.

Reads, as text, the reference's B-spline known-answer harness
(src/libs/BS/TEST_BS/: knot.dat, int_out, int_inp1, quadr_out) and the
Gauss-Legendre table of src/libs/BS/gauss.f90, and writes
tests/golden/test_bs_golden.json.  Run from the repository root:

    python tests/golden/make_golden.py /path/to/jagot-bsr
    BSR_REFERENCE=/path/to/jagot-bsr python tests/golden/make_golden.py

The output is committed; tests never read the reference tree at run time.
"""
import json
import os
import re
import sys


def parse_knot_dat(text):
    """knot.dat grid_type 0 header: ks, ns, z, h, hmax, rmax (define_grid.f90:59-64)."""
    lines = text.splitlines()
    vals = [lines[i].split()[0] for i in range(6)]
    return {"ks": int(vals[0]), "ns": int(vals[1]), "z": float(vals[2]),
            "h": float(vals[3]), "hmax": float(vals[4]), "rmax": float(vals[5])}


def parse_int_out(text):
    """int_out: one header line per integral followed by one line per route."""
    out = []
    cur = None
    head = re.compile(r"^([RNMTVWQ])\s*(-?\d+)\(\s*(\w+),\s*(\w+);\s*(\w+),\s*(\w+)\)=\s*(\S+)")
    for line in text.splitlines():
        m = head.match(line)
        if m:
            cur = {"int": m.group(1), "k": int(m.group(2)),
                   "orbs": [m.group(3), m.group(4), m.group(5), m.group(6)],
                   "routes": {}}
            out.append(cur)
            continue
        parts = line.split()
        if cur is not None and len(parts) == 3:
            val = float(parts[0].replace("D", "E"))
            cur["routes"][parts[2]] = val
    return out


def parse_int_inp1(text):
    """int_inp1: analytic hydrogenic integrals as S1/S2 (times Z for R^k, test_bs.f90:326-328)."""
    out = []
    pat = re.compile(r"^([RNMTVWQ])\s*(-?\d+)\(\s*(\w+),\s*(\w+);\s*(\w+),\s*(\w+)\)=\s*(\S+)\s+(\S+)")
    for line in text.splitlines():
        m = pat.match(line)
        if not m:
            continue
        s1 = float(m.group(7).replace("d", "e").replace("D", "E"))
        s2 = float(m.group(8).replace("d", "e").replace("D", "E"))
        out.append({"int": m.group(1), "k": int(m.group(2)),
                    "orbs": [m.group(3), m.group(4), m.group(5), m.group(6)],
                    "ratio": s1 / s2})
    return out


def parse_quadr_out(text):
    """quadr_out 'accuracy of orthogonality' block: <i|j> - delta_ij per same-l pair."""
    out = []
    on = False
    for line in text.splitlines():
        if "accuracy of orthogonality" in line:
            on = True
            continue
        if "accuracy of <r^m>" in line:
            break
        parts = line.split()
        if on and len(parts) == 3:
            out.append({"a": parts[0], "b": parts[1], "err": float(parts[2].replace("D", "E"))})
    return out


def parse_gauss_table(text, k):
    """The k-point node/weight table of gauss.f90 (CASE (k) block)."""
    blk = re.search(r"CASE \(%d\)(.*?)(CASE|END SELECT)" % k, text, re.S).group(1)
    xs, ws = {}, {}
    for m in re.finditer(r"([xw])\((\d+)\)\s*=\s*([0-9.eEdD+-]+)", blk):
        v = float(m.group(3).replace("d", "e").replace("D", "E"))
        (xs if m.group(1) == "x" else ws)[int(m.group(2))] = v
    return [xs[i] for i in range(1, k + 1)], [ws[i] for i in range(1, k + 1)]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BSR_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <jagot/bsr source tree> (or set BSR_REFERENCE)")
    tb = os.path.join(ref, "src/libs/BS/TEST_BS")
    read = lambda p: open(p).read()
    golden = {
        "source": "jagot/bsr src/libs/BS/TEST_BS (knot.dat, int_out, int_inp1, quadr_out) "
                  "and src/libs/BS/gauss.f90",
        "knot": parse_knot_dat(read(os.path.join(tb, "knot.dat"))),
        "int_out": parse_int_out(read(os.path.join(tb, "int_out"))),
        "int_inp1": parse_int_inp1(read(os.path.join(tb, "int_inp1"))),
        "quadr_orth": parse_quadr_out(read(os.path.join(tb, "quadr_out"))),
        "gauss": {},
    }
    gtext = read(os.path.join(ref, "src/libs/BS/gauss.f90"))
    for k in (4, 8, 10):
        x, w = parse_gauss_table(gtext, k)
        golden["gauss"][str(k)] = {"x": x, "w": w}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "test_bs_golden.json")
    with open(dst, "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", dst, "with", len(golden["int_out"]), "int_out integrals")


if __name__ == "__main__":
    main()
