"""Load the committed golden fixtures (made by tests/golden/make_golden.py)."""
import glob
import os

import numpy as np

from pyscfad_b200.synthetic import TriplesInputs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEYS = ("mo_energy", "t1", "t2", "ovoo", "ovov", "ovvv", "fvo")
LNO_PREFIX = "lno_"
DF_PREFIX = "df_"
SLICE_PREFIX = "slice_"   # one virtual slice of a benchmark-size problem (tests/golden/make_slices.py)


def _all():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def names():
    """Canonical (T) fixtures."""
    return [n for n in _all() if not n.startswith((LNO_PREFIX, DF_PREFIX, SLICE_PREFIX))]


def df_names():
    """Canonical (T) fixtures whose inputs are given as DF factors (Lov, packed Lvv)."""
    return [n for n in _all() if n.startswith(DF_PREFIX)]


def lno_names():
    """LNO fragment (T) fixtures (projector mat on the first occupied index)."""
    return [n for n in _all() if n.startswith(LNO_PREFIX)]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    inp = TriplesInputs(*[np.ascontiguousarray(z["in_" + k]) for k in KEYS])
    grads = {k: z["grad_" + k] for k in KEYS}
    if name.startswith(LNO_PREFIX):
        grads["mat"] = z["grad_mat"]
    return inp, float(z["e"]), grads, z
