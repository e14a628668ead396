"""Generates tests/golden/transport_golden.npz from the reference's own
transport element (iga::BuildTransportElement, solvers/cpu/include/
TransportElement.hpp:213-260, compiled unmodified into
oracle/_ref/libtfiga_ref.so).  Run where the reference build exists:

    make -C oracle ref && python tests/golden/make_transport_golden.py

Elements: the unit identity-extraction element of the reference's element
known-answer test (solvers/cpu/tests/test_navier_stokes.cpp:21-36) and its
curved variant, with a smooth nodal velocity field, under two parameter
sets (advective with SUPG and artificial diffusion; a pure reaction-diffusion
set with zero velocity, where the SUPG weight vanishes).  Stored: the full
left and previous matrices of each case.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle  # noqa: E402
from tests.golden.make_element_golden import curved, unit_element  # noqa: E402

PARAMS = {
    "advective": {"diffusion": 1e-3, "vplus": 0.8, "kplus": 0.3, "kminus": 0.05, "detach_plus": 0.2,
                  "dt": 0.01, "artificial_diffusion": 0.02},
    "reaction": {"diffusion": 0.05, "vplus": 1.0, "kplus": 0.5, "kminus": 0.25, "detach_plus": 0.125,
                 "dt": 0.1, "artificial_diffusion": 0.0},
}


def velocity(X, still=False):
    if still:
        return np.zeros((X.shape[0], 3))
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    return np.stack([0.2 + 0.1 * y, -0.05 * z + 0.02 * x, 1.0 - 0.3 * x * x], axis=1)


def cases():
    C, X = unit_element()
    for geometry, Xg in (("unit", X), ("curved", curved(X))):
        for name, p in PARAMS.items():
            yield f"{geometry}_{name}", C, Xg, velocity(Xg, still=(name == "reaction")), p


def main():
    out = {}
    for key, C, X, vel, p in cases():
        left, previous = oracle.transport_element(C, X, vel, p, use_ref=True)
        out[f"{key}_left"] = left
        out[f"{key}_previous"] = previous
    np.savez_compressed(Path(__file__).with_name("transport_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
