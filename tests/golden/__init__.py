"""Committed golden fixtures (see make_golden.py for how each was produced)."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load(name):
    with np.load(os.path.join(HERE, name + ".npz")) as f:
        return {k: f[k] for k in f.files}
