"""The CPU oracle (oracle/src) against the reference's own full-precision
output (tests/golden, generated from the compiled reference)."""
import numpy as np
import pytest

from tests._cases import case_setup, load_cases, parse_golden, profile_path

CASES = {k: v for k, v in load_cases().items() if v["binary"] == "iga_ref_3d" and v["mode"] == "prop"}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference(name, oracle_mod):
    c = CASES[name]
    th, ph, p = case_setup(c["args"])
    rows, steps = oracle_mod.fan_3d(profile_path(c["seed"]), th, ph, **p)
    ref, ref_steps = parse_golden(name)
    assert steps.shape == ref_steps.shape
    np.testing.assert_array_equal(steps, ref_steps)
    assert rows.shape == ref.shape
    # Same algorithm, same operation order, same libm: bit-identical.
    np.testing.assert_array_equal(rows, ref)


def test_oracle_threads_match_serial(oracle_mod):
    c = CASES["3d_noamp"]
    th, ph, p = case_setup(c["args"])
    a, sa = oracle_mod.fan_3d(profile_path(c["seed"]), th, ph, **p)
    b, sb = oracle_mod.fan_3d(profile_path(c["seed"]), th, ph, **dict(p, n_threads=4))
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(sa, sb)
