"""Vertex-centred ENO prolongation: a second, independent restatement.

CarpetLib's prolongate_3d_real8_eno is Fortran (prolongate_3d_real8_eno.F90)
and this image has no Fortran compiler, so the C oracle's restatement
(oracle/cgx_oracle.c, which the GPU kernels match bit for bit) cannot be
pinned to a compiled build of it.  This file restates the routine a second
time, in plain Python, line by line from the Fortran source, and checks the
two restatements against each other bit for bit on every parity case of the
fine point, on random regions and on fields that drive every branch of the
limiter; it also checks the properties the routine guarantees by
construction.  (The cell-centred ENO is C++ in the reference and is pinned
to its compiled build in tests/test_oracle.py.)

Source lines followed:
  eno1d                  F90:23-76
  the fine-point loop    F90:187-279 (parity cases 0, 1, 10, 11, 100, 101,
                         110, 111; x innermost, then y, then z)
Python floats are IEEE binary64 with round-to-nearest and no contraction,
and every expression keeps the Fortran source's left-to-right order, so the
result is the canonical (uncontracted) evaluation.
"""
import numpy as np
import pytest

from oracle import cases
from oracle.binding import Port, box_sizes

EIGHTH, HALF = 1.0 / 8.0, 0.5


def eno1d(q1, q2, q3, q4):
    """F90:23-76 -- ENO2-limited quadratic between q2 and q3"""
    diffleft = (q1 + q3) - 2.0 * q2
    diffright = (q2 + q4) - 2.0 * q3
    if abs(diffleft) < abs(diffright):
        r = EIGHTH * ((-q1 + 6.0 * q2) + 3.0 * q3)   # the left quadratic
    else:
        r = EIGHTH * ((3.0 * q2 + 6.0 * q3) - q4)    # the right quadratic
    if (r - q2) * (q3 - r) < 0.0 or diffleft * diffright <= 0.0:
        r = HALF * (q2 + q3)                         # linear interpolation
    return r


def prolongate_eno_py(src, srcbbox, dst, dstbbox, reg):
    """F90:187-279 for refinement factor 2 (arrays (nz, ny, nx_pad), x fastest)"""
    S = lambda i, j, k: float(src[k, j, i])
    ext = box_sizes(reg)
    soff = [(reg[d] - srcbbox[d]) // dstbbox[6 + d] for d in range(3)]
    doff = [(reg[d] - dstbbox[d]) // dstbbox[6 + d] for d in range(3)]
    for k in range(ext[2]):
        for j in range(ext[1]):
            for i in range(ext[0]):
                i0, fi = divmod(soff[0] + i, 2)
                j0, fj = divmod(soff[1] + j, 2)
                k0, fk = divmod(soff[2] + k, 2)
                # the four coarse points of an odd axis are base - 1 .. base + 2
                xl = lambda jj, kk: eno1d(*(S(i0 - 1 + a, jj, kk) for a in range(4)))
                case = fi + 10 * fj + 100 * fk
                if case == 0:
                    v = S(i0, j0, k0)
                elif case == 1:
                    v = xl(j0, k0)
                elif case == 10:
                    v = eno1d(*(S(i0, j0 - 1 + a, k0) for a in range(4)))
                elif case == 11:
                    v = eno1d(*(xl(j0 - 1 + jj, k0) for jj in range(4)))
                elif case == 100:
                    v = eno1d(*(S(i0, j0, k0 - 1 + a) for a in range(4)))
                elif case == 101:
                    v = eno1d(*(xl(j0, k0 - 1 + kk) for kk in range(4)))
                elif case == 110:
                    v = eno1d(*(eno1d(*(S(i0, j0 - 1 + a, k0 - 1 + kk) for a in range(4)))
                                for kk in range(4)))
                else:  # 111: x lines, then y over each z, then z
                    tmp1 = [[xl(j0 - 1 + jj, k0 - 1 + kk) for kk in range(4)] for jj in range(4)]
                    tmp2 = [eno1d(*(tmp1[jj][kk] for jj in range(4))) for kk in range(4)]
                    v = eno1d(*tmp2)
                dst[doff[2] + k, doff[1] + j, doff[0] + i] = v


@pytest.fixture(scope="module")
def port():
    return Port()


@pytest.mark.parametrize("kind", ["normal", "steps", "smooth", "mixed"])
def test_c_oracle_equals_python_restatement(port, kind):
    """both restatements of the Fortran routine agree bit for bit"""
    rng = np.random.default_rng({"normal": 1, "steps": 2, "smooth": 3, "mixed": 4}[kind])
    cases_seen = set()
    for _ in range(12):
        c = cases.vc_prolong_case(rng, 3, max_ext=7, kind=kind, reach=(1, 2))
        got = c["dst"].copy()
        port.prolongate_3d_eno(c["src"], c["srcbbox"], got, c["dstbbox"], c["reg"])
        want = c["dst"].copy()
        prolongate_eno_py(c["src"], c["srcbbox"], want, c["dstbbox"], c["reg"])
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), kind
        reg, sb = c["reg"], c["srcbbox"]
        for d in range(3):
            cases_seen.add((d, (reg[d] - sb[d]) // reg[6 + d] % 2))
    assert len(cases_seen) == 6  # odd and even region starts on every axis


def test_eno1d_branches_and_bounds():
    """every branch of the limiter is taken, and the result always lies
    between the two middle values (F90:62-73)"""
    rng = np.random.default_rng(7)
    seen = set()
    for _ in range(20000):
        q = rng.standard_normal(4) * rng.choice([1.0, 1e-3, 1e3])
        dl = (q[0] + q[2]) - 2.0 * q[1]
        dr = (q[1] + q[3]) - 2.0 * q[2]
        r = eno1d(*q)
        lin = HALF * (q[1] + q[2])
        if r == lin and not (dl * dr > 0.0 and r == (EIGHTH * ((-q[0] + 6.0 * q[1]) + 3.0 * q[2])
                                                 if abs(dl) < abs(dr) else
                                                 EIGHTH * ((3.0 * q[1] + 6.0 * q[2]) - q[3]))):
            seen.add("linear")
        else:
            seen.add("left" if abs(dl) < abs(dr) else "right")
        assert min(q[1], q[2]) <= r <= max(q[1], q[2])
    assert seen == {"left", "right", "linear"}


def test_linear_fields_are_reproduced(port):
    """on a field linear along every axis the second differences vanish, the
    limiter takes the linear branch everywhere, and with dyadic values every
    fine point is the exact average of its coarse neighbours"""
    rng = np.random.default_rng(11)
    for _ in range(6):
        c = cases.vc_prolong_case(rng, 3, max_ext=7, reach=(1, 2))
        src = c["src"]
        nz, ny, nx = src.shape
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        a = rng.integers(-8, 8, 4)
        src[...] = a[0] + a[1] * x + a[2] * y + a[3] * z
        got = c["dst"].copy()
        port.prolongate_3d_eno(src, c["srcbbox"], got, c["dstbbox"], c["reg"])
        reg, sb = c["reg"], c["srcbbox"]
        ext = box_sizes(reg)
        dof = [(reg[d] - c["dstbbox"][d]) // reg[6 + d] for d in range(3)]
        for k in range(ext[2]):
            for j in range(ext[1]):
                for i in range(ext[0]):
                    # the fine point's position in coarse index units
                    p = [((reg[d] - sb[d]) // reg[6 + d] + (i, j, k)[d]) / 2.0 for d in range(3)]
                    want = a[0] + a[1] * p[0] + a[2] * p[1] + a[3] * p[2]
                    assert got[dof[2] + k, dof[1] + j, dof[0] + i] == want


def test_result_bounded_by_the_surrounding_coarse_values(port):
    """each 1-D pass stays between its two middle inputs, so a fine point
    stays within the range of the 2 x 2 x 2 coarse points around it: the
    property the routine exists for (positivity of a density, F90:3-20)"""
    rng = np.random.default_rng(13)
    for kind in ("normal", "steps", "mixed"):
        for _ in range(6):
            c = cases.vc_prolong_case(rng, 3, max_ext=7, kind=kind, reach=(1, 2))
            got = c["dst"].copy()
            port.prolongate_3d_eno(c["src"], c["srcbbox"], got, c["dstbbox"], c["reg"])
            reg, sb, db = c["reg"], c["srcbbox"], c["dstbbox"]
            ext = box_sizes(reg)
            soff = [(reg[d] - sb[d]) // reg[6 + d] for d in range(3)]
            dof = [(reg[d] - db[d]) // reg[6 + d] for d in range(3)]
            src = c["src"]
            for k in range(ext[2]):
                for j in range(ext[1]):
                    for i in range(ext[0]):
                        b = [divmod(soff[d] + (i, j, k)[d], 2) for d in range(3)]
                        nb = src[b[2][0]:b[2][0] + 1 + b[2][1], b[1][0]:b[1][0] + 1 + b[1][1],
                                 b[0][0]:b[0][0] + 1 + b[0][1]]
                        v = got[dof[2] + k, dof[1] + j, dof[0] + i]
                        assert nb.min() <= v <= nb.max(), (kind, i, j, k)
