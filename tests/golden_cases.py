"""Loads the golden fixtures (outputs of the reference itself, see
tests/golden/make_golden.py) and regenerates their inputs from the seeds."""
import json
import os

import numpy as np

from make_golden import CASES, TEXT_CASES, BETAS, pairs_sha, synth_case  # noqa: F401

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))

SYNTH = [k for k, v in MANIFEST.items() if isinstance(v, dict) and v.get("kind") == "synth"]
TEXT = [k for k, v in MANIFEST.items() if isinstance(v, dict) and v.get("kind") == "text"]
SMALL = [k for k in SYNTH if k not in ("c1", "c2", "hubs")]


def expected(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def inputs(name):
    """Per-layer raw pairs of a synthetic case, checked against the stored hash."""
    layers = synth_case(name)
    assert pairs_sha(layers) == MANIFEST[name]["pairs_sha256"], \
        f"{name}: regenerated input differs from the one the fixture was made from"
    return layers


def texts(name):
    return MANIFEST[name]["texts"]
