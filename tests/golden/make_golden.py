"""Extract the CarpetProlongateTest golden error norms into a fixture.

Reads the reference's own testsuite (CarpetProlongateTest/test/*.par and the
stored carpetprolongatetest-errornorm..asc outputs, plus the tolerances of
CarpetProlongateTest/test/test.ccl) and writes
tests/golden/prolongatetest_errornorms.json.  Run it where the reference
sources are present:

    python tests/golden/make_golden.py /root/reference
"""
import json
import os
import re
import sys


def par_value(text, key, default=None):
    m = re.search(r"^\s*" + re.escape(key) + r"\s*=\s*\"?([^\"\n#]+)\"?", text, re.M)
    return m.group(1).strip() if m else default


def main(ref):
    tdir = os.path.join(ref, "CarpetProlongateTest", "test")
    ccl = open(os.path.join(tdir, "test.ccl")).read()
    tols = {}
    for name, body in re.findall(r"TEST\s+(\S+)\s*\{([^}]*)\}", ccl):
        t = {}
        for k in ("ABSTOL", "RELTOL"):
            m = re.search(k + r"\s+(\S+)", body)
            if m:
                t[k.lower()] = float(m.group(1))
        tols[name] = t
    out = []
    for fn in sorted(os.listdir(tdir)):
        if not fn.endswith(".par"):
            continue
        name = fn[:-4]
        asc = os.path.join(tdir, name, "carpetprolongatetest-errornorm..asc")
        if not os.path.exists(asc):
            continue
        par = open(os.path.join(tdir, fn)).read()
        vals = [l.split() for l in open(asc) if l.strip() and not l.startswith("#")]
        entry = dict(
            test=name,
            errornorm=float(vals[0][-1]),
            centering=par_value(par, "Carpet::refinement_centering", "vertex"),
            prolongation_order_space=int(par_value(par, "Carpet::prolongation_order_space", "1")),
            prolongation_type=par_value(par, "CarpetProlongateTest::prolongation_type", "Lagrange"),
            ghost_size=int(par_value(par, "driver::ghost_size", "0")),
            power_x=int(par_value(par, "CarpetProlongateTest::power_x", "0")),
            power_y=int(par_value(par, "CarpetProlongateTest::power_y", "0")),
            power_z=int(par_value(par, "CarpetProlongateTest::power_z", "0")),
            dx=float(par_value(par, "CoordBase::dx", "0")),
            radius=float(par_value(par, "CarpetRegrid2::radius_1[1]", "0")),
            use_higher_order_restriction=par_value(
                par, "CarpetLib::use_higher_order_restriction", "no"),
            source=os.path.relpath(asc, ref),
            **tols.get(name, {}),
        )
        out.append(entry)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "prolongatetest_errornorms.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} entries to {dst}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
