"""roofline.json (the FLOP counts bench.py divides by) reproduces from the
operation-counting build of the oracle restatement."""
import json
import os

from oracle.opcount import make_roofline

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_roofline_counts_reproduce():
    with open(os.path.join(ROOT, "roofline.json")) as f:
        committed = json.load(f)
    fresh = make_roofline.compute()
    assert fresh["weights"] == committed["weights"]
    assert fresh["variants"] == committed["variants"]
    # the absorption model is about a fifth of the FP64 amplitude step
    v = committed["variants"]
    assert 0.1 < (v["fp64_amp"] - v["fp32c_amp"]) / v["fp64_amp"] < 0.4
