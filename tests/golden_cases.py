"""Loader for the committed golden vectors (tests/golden/)."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load():
    with open(os.path.join(HERE, "reference_outputs.json")) as f:
        meta = json.load(f)
    arrays = dict(np.load(os.path.join(HERE, "reference_outputs.npz")))
    return meta, arrays
