"""Reference outputs for the CrabCav, RFMult and IdealWig elements (oracle/_ref).

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_elem_extra_golden.py

Each case is one element, written with the engine's lattice writer, read and tracked for one turn
by the reference library on the 16 particles of make_golden.element_particles().  Crab cavities
are switched on (the reference's constructor leaves them off); the radiating wiggler has
radiation switched on.  Writes elements_extra.npz: elem_in and elem_<case> per case.
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)


def cases(A):
    e = A.elem
    return {
        "crabcav": [e(A.CRABCAV, "CC", 0.4, f=[1.2, 0.8, 476.314e6 * 6, 0.1, 3000, 0, 0], flags=1)],
        "crabcav_thin": [e(A.CRABCAV, "CC", 0.0, f=[0.5, -0.3, 476.314e6 * 3, -0.2, 3000, 0, 0], flags=1)],
        "rfmult": [e(A.RFMULT, "RM", 0.2, f=[476.314e6 * 3, 0.3, 3000, 0, 0], max_npole=3,
                     poly_b=[1e-4, 0.2, 3.0], poly_a=[0.0, 0.05, 0.5])],
        "idealwig_h": [e(A.IDEALWIG, "W", 1.5, nslice=20, f=[0.05, 1.2, 0, 3000])],
        "idealwig_v": [e(A.IDEALWIG, "W", 1.5, nslice=20, f=[0.05, 1.2, 1, 3000])],
        "idealwig_rad": [e(A.IDEALWIG, "W", 1.5, nslice=20, f=[0.05, 0.1, 0, 3000], flags=1)],
    }


def main():
    import oracle as O
    import make_golden as MG
    A = importlib.import_module("accel-plus_b200")
    r0 = MG.element_particles()
    out = {"elem_in": r0}
    for name, elems in cases(A).items():
        fd, path = tempfile.mkstemp(suffix=".lat")
        os.close(fd)
        A.write_lattice(path, elems)
        line = O.RefLine(path)
        os.unlink(path)
        if name.startswith("crabcav"):
            line.set_crab(True)
        if name == "idealwig_rad":
            line.set_flags(rad=1)
        r = r0.copy()
        line.track(r, 1)
        out[f"elem_{name}"] = r
        print(name, np.abs(r - r0).max())
    np.savez_compressed(os.path.join(HERE, "elements_extra.npz"), **out)


if __name__ == "__main__":
    main()
