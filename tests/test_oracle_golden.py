"""The CPU oracle against the reference's own results (CPU, no GPU).

Pins the oracle: known answers asserted by the reference's tests, and the
printed results of this repository's drivers built on the reference's
sequential backend (tests/golden/golden.json, tests/golden/make_golden.py).
"""

import os
import re
import tempfile

import pytest

from tests.apprun import (assert_lines_close, clover_deck_test1, result_lines, run_app,
                          run_exe)


def test_poisson_mb_oracle_matches_reference(golden):
    out, _ = run_app("poisson_mb", "oracle")
    want = golden["reference_runs"]["poisson_mb_default"]["lines"]
    got = result_lines(out)
    # residual history: max reductions, bit-identical; checksum is a sum
    assert got[:-1] == want[:-1]
    assert_lines_close(got[-1:], want[-1:], 1e-13)


def test_poisson_mb_3x3_oracle_matches_reference(golden):
    g = golden["reference_runs"]["poisson_mb_3x3"]
    out, _ = run_app("poisson_mb", "oracle", g["args"])
    assert_lines_close(result_lines(out), g["lines"], 1e-13)


@pytest.mark.parametrize("case", ["opsunit_default", "opsunit_29x17"])
def test_opsunit_oracle_matches_reference(golden, case):
    g = golden["reference_runs"][case]
    out, _ = run_app("opsunit", "oracle", g["args"])
    got = [l for l in result_lines(out) if l.split()[0] in ("sums", "min", "max", "count",
                                                             "fetch_b")]
    assert_lines_close(got, g["lines"], 1e-14)


def test_reference_poisson_known_answer_on_oracle(golden):
    out = run_exe("ref_poisson", "oracle")
    v = float(re.search(r"Total error: (\S+)", out).group(1))
    want = golden["known_answers"]["ref_poisson_default_total_error"]["value"]
    assert abs(v - want) <= 1e-12 * want
    assert "PASSED" in out


def test_reference_cloverleaf_test1_on_oracle(golden):
    d = tempfile.mkdtemp(prefix="clover_t1_")
    with open(os.path.join(d, "clover.in"), "w") as f:
        f.write(clover_deck_test1())
    out = run_exe("cloverleaf", "oracle", cwd=d)
    assert "This test is considered PASSED" in out
    m = re.search(r"within (\S+) %", out)
    assert float(m.group(1)) < 1e-9


HEAT_KEYS = ("fp64", "mixed", "compare")


@pytest.mark.parametrize("case", ["heat_cg_128", "heat_cg_96_fixed"])
def test_heat_cg_oracle_matches_reference(golden, case):
    """CG heat conduction (FP64 CG and FP32-inner / FP64-refinement): the
    oracle's iteration counts, residuals and checksums against the same
    driver on the reference's sequential backend."""
    g = golden["reference_runs"][case]
    out, _ = run_app("heat_cg", "oracle", g["args"])
    assert_lines_close(result_lines(out, HEAT_KEYS), g["lines"], 1e-11)
