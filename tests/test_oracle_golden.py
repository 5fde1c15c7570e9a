"""The C restatement against golden digests of the reference's own outputs
(tests/golden/ref_digests.json, made by tests/golden/make_golden.py from the
reference sources compiled unmodified).  Runs without the reference sources."""
import hashlib
import json
import os

import pytest

from lenia_cases import VARIANTS, as_oracle, four_channels, two_channel_div_flow, variant
from oracle.oracle import RestateOracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_digests.json")


def digest(a) -> str:
    return hashlib.sha256(a.astype("<f4").tobytes()).hexdigest()


def load():
    with open(GOLDEN) as f:
        return json.load(f)


def workload(name):
    if name == "div_flow_2ch":
        return two_channel_div_flow()
    if name == "four_channels":
        return four_channels()
    return variant(name)


@pytest.mark.parametrize("name", sorted(VARIANTS) + ["div_flow_2ch", "four_channels"])
def test_restatement_matches_reference_digests(oracle_built, name):
    gold = load()
    rec = gold["cases"][name]
    wl = workload(name)
    p, ks = as_oracle(wl)
    ora = RestateOracle(p, ks, fft_mode="c2c")
    ora.set_state(A=wl.A0.ravel())
    for step in range(gold["steps"]):
        ora.step(1)
        for f in gold["fields"]:
            assert digest(ora.get(f)) == rec[step][f], f"{name} step {step} field {f}"
