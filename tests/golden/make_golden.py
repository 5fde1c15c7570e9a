"""Writes tests/golden/ref_digests.json: SHA-256 digests of the reference's own
step outputs (oracle/_ref, the reference sources compiled unmodified) for the
mode variants of tests/lenia_cases.py, after each of two steps, plus a few
sample values.  Run here, where the reference sources exist:

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lenia_cases import VARIANTS, as_oracle, four_channels, two_channel_div_flow, variant  # noqa: E402
from oracle.oracle import RefOracle  # noqa: E402

FIELDS = ["A", "V", "GA", "SUM", "H", "U_SUM", "BACK", "MU", "U"]


def digest(a) -> str:
    return hashlib.sha256(a.astype("<f4").tobytes()).hexdigest()


def cases():
    for name in sorted(VARIANTS):
        yield name, variant(name)
    yield "div_flow_2ch", two_channel_div_flow()
    yield "four_channels", four_channels()


def main():
    out = {"steps": 2, "fields": FIELDS, "cases": {}}
    for name, wl in cases():
        p, ks = as_oracle(wl)
        ref = RefOracle(p, ks)
        ref.set_state(A=wl.A0.ravel())
        rec = []
        for step in range(2):
            ref.step(1)
            rec.append({f: digest(ref.get(f)) for f in FIELDS})
            a = ref.get("A")
            rec[-1]["A_samples"] = [float(a[i]) for i in range(0, a.size, a.size // 7)]
        out["cases"][name] = rec
    with open(os.path.join(HERE, "ref_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
