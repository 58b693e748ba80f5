"""Fields where bound states cross a fixed energy (molscat_b200/field.py,
FIELD's search in fld.driver.f).

Pinned through an exact equivalence: shifting every channel threshold by
s*F (s = +-1 cm-1 per unit field) is the same as moving the energy by -s*F,
so at energy E the crossings lie at F = s*(E - E_k), with E_k the
reference's printed bound-basic1 energies (examples/output/bound-basic1.output,
JTOT=1 block 2, states 4 and 5).  s = +1 makes the count fall with the field,
s = -1 makes it rise: both of FIELD's directions."""
import dataclasses

import numpy as np
import pytest

from molscat_b200.bound import bisect_steps
from molscat_b200.field import FieldProblem, field_node_counts, find_fields, find_fields_converged
from test_bound import REF_TOL_CM, TOL_CM, basic1, oracle_counts, oracle_eval  # noqa: F401  (fixture)

E_CM = -3.0


def field_problem(basic1, sign):
    g, sysm, bp = basic1
    c0 = bp.coupling

    def coupling_at(f):
        # every other coupling field (NVLBLK, IV, IVLFL, NCONST, ...) carries over
        return dataclasses.replace(c0, eint=c0.eint + sign * f * sysm.cm2ru)

    fp = FieldProblem(coupling_at, bp.seg_out, bp.seg_in, E_CM * sysm.cm2ru, "LDMD")
    s = g["system"]
    # the field window that maps onto the golden energy window [emin, emax]
    ends = sorted([sign * (E_CM - s["emin_cm"]), sign * (E_CM - s["emax_cm"])])
    want = sorted(sign * (E_CM - st["energy_cm"]) for st in g["states"])
    return fp, ends, want


def oracle_field_counts(fp, fields):
    """The oracle's count at each field (BOUND's count with that field's coupling)."""
    from molscat_b200.bound import BoundProblem
    out = []
    for f in fields:
        c = fp.coupling_at(float(f))
        bp = BoundProblem(c, fp.seg_out, fp.seg_in, fp.prop,
                          y_out0=lambda e, c=c: fp.y_out0(c), y_in0=lambda e, c=c: fp.y_in0(c))
        out.append(int(oracle_counts(bp, [fp.ered])[0]))
    return np.array(out)


def test_bisect_steps_both_directions():
    steps = np.array([-0.7, 0.2, 0.9])
    up = bisect_steps(lambda x: np.searchsorted(steps, x), -1.0, 1.0, 0, 3, 1e-10)
    down = bisect_steps(lambda x: 3 - np.searchsorted(steps, x), -1.0, 1.0, 3, 0, 1e-10)
    assert [k for k, *_ in up] == [0, 1, 2] and [k for k, *_ in down] == [0, 1, 2]
    assert np.allclose([x for _, x, *_ in up], steps, atol=1e-10)
    # falling count: the step between k + 1 and k is the (3 - k)-th level from the top
    assert np.allclose([x for _, x, *_ in down], steps[::-1], atol=1e-10)


@pytest.mark.parametrize("sign", [1, -1])
def test_oracle_fields_match_reference_energies(basic1, sign):
    fp, (fmin, fmax), want = field_problem(basic1, sign)
    found = find_fields(fp, fmin, fmax, TOL_CM, counter=oracle_field_counts)
    got = sorted(f for _, f, _, _ in found)
    assert len(got) == len(want)
    for f, w in zip(got, want):
        assert abs(f - w) < REF_TOL_CM, (f, w)


@pytest.mark.gpu
def test_gpu_field_counts_equal_oracle(basic1):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    fp, (fmin, fmax), want = field_problem(basic1, 1)
    probe = [fmin, fmax] + [w + d for w in want for d in (-1e-6, 1e-6)]
    assert np.array_equal(field_node_counts(fp, probe)[0], oracle_field_counts(fp, probe))
    found = find_fields(fp, fmin, fmax, TOL_CM)
    got = sorted(f for _, f, _, _ in found)
    assert len(got) == len(want)
    for f, w in zip(got, want):
        assert abs(f - w) < REF_TOL_CM, (f, w)
    # the same fields as the oracle's search: both bisect the same midpoints,
    # so equal counts at every midpoint give identical fields
    ora = sorted(f for _, f, _, _ in find_fields(fp, fmin, fmax, TOL_CM, counter=oracle_field_counts))
    assert got == ora


def oracle_field_eval(fp, fields):
    from molscat_b200.bound import BoundProblem
    cnt, eig = [], []
    for f in fields:
        c = fp.coupling_at(float(f))
        bp = BoundProblem(c, fp.seg_out, fp.seg_in, fp.prop,
                          y_out0=lambda e, c=c: fp.y_out0(c), y_in0=lambda e, c=c: fp.y_in0(c))
        a, b = oracle_eval(bp, [fp.ered])
        cnt.append(int(a[0]))
        eig.append(float(b[0]))
    return np.array(cnt), np.array(eig)


@pytest.mark.parametrize("sign", [1, -1])
def test_oracle_converged_fields_match_reference_energies(basic1, sign):
    fp, (fmin, fmax), want = field_problem(basic1, sign)
    found, rounds = find_fields_converged(fp, fmin, fmax, TOL_CM, evaluate=oracle_field_eval)
    got = sorted(f for _, f, _, _ in found)
    assert len(got) == len(want)
    for f, w in zip(got, want):
        assert abs(f - w) < REF_TOL_CM, (f, w)
    assert rounds < 25


@pytest.mark.gpu
def test_gpu_converged_fields_equal_oracle(basic1):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    fp, (fmin, fmax), want = field_problem(basic1, 1)
    got = sorted(f for _, f, _, _ in find_fields_converged(fp, fmin, fmax, TOL_CM)[0])
    ora = sorted(f for _, f, _, _ in find_fields_converged(fp, fmin, fmax, TOL_CM, evaluate=oracle_field_eval)[0])
    assert len(got) == len(want) == len(ora)
    for f, o in zip(got, ora):
        assert abs(f - o) <= 1e-9 * abs(o), (f, o)
