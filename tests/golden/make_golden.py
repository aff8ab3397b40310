"""Regenerates the golden discrete-ordinate fixtures from the reference's own run logs.

The reference prints its SN ordinates (AngularSpace.f90:52-118, 16 significant digits) at the
start of every run.  This script parses those tables out of three shipped logs and writes them as
plain text next to itself:

  ordinates_L11.txt  288 x 3  validation/photons_incident/water_tank_6MeV/lb.out   (PNSCATTERING 11)
  ordinates_L7.txt   128 x 3  examples/three_beam_water_tank/lb.out                (PNSCATTERING 7)
  mu_slab_L15.txt     16      validation/electrons_incident/Al_521keV_0deg/lb.out  (slab, 16-point GL)

Run from anywhere:  python tests/golden/make_golden.py <Lionbolt source root>
"""
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIONBOLT_REFERENCE") or sys.exit(
    "usage: make_golden.py <Lionbolt source root> (or set LIONBOLT_REFERENCE)")
HERE = os.path.dirname(os.path.abspath(__file__))


def first_table(path, slab=False):
    lines = open(path, encoding="utf-8").read().splitlines()
    start = next(i for i, l in enumerate(lines) if l.strip().startswith("Ordinates"))
    rows = []
    pat3 = re.compile(r"^\s*(\d+)\s*\)\s*\(\s*(\S+),\s*(\S+),\s*(\S+)\s*\)")
    pat1 = re.compile(r"^\s*(\d+)\s*\)\s*(\S+)\s*$")
    for l in lines[start + 3:]:
        m = (pat1 if slab else pat3).match(l)
        if not m:
            break
        rows.append([float(v) for v in m.groups()[1:]])
    return rows


def main():
    jobs = [
        ("ordinates_L11.txt", "validation/photons_incident/water_tank_6MeV/lb.out", False, 288),
        ("ordinates_L7.txt", "examples/three_beam_water_tank/lb.out", False, 128),
        ("mu_slab_L15.txt", "validation/electrons_incident/Al_521keV_0deg/lb.out", True, 16),
    ]
    for out, src, slab, n in jobs:
        rows = first_table(os.path.join(REF, src), slab)
        assert len(rows) == n, (src, len(rows))
        with open(os.path.join(HERE, out), "w") as f:
            f.write(f"# parsed from {src} (reference run log), {n} rows\n")
            for r in rows:
                f.write(" ".join(f"{v:.16f}" for v in r) + "\n")
        print(out, len(rows))


if __name__ == "__main__":
    main()
