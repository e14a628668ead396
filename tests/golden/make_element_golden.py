"""Generates tests/golden/element_golden.npz from the reference's own element
code (oracle/_ref/libtfiga_ref.so, compiled unmodified from the reference's
NavierStokesElement.hpp).  Run where the reference build exists:

    make -C oracle ref && python tests/golden/make_element_golden.py

The elements and states are those of the reference's known-answer test
(solvers/cpu/tests/test_navier_stokes.cpp:21-36 and :191-245): the unit
identity-extraction element and its curved variant, with the same nodal
state, previous state and parameters.  Stored: the full negative residual
and every 16th Jacobian row, steady and transient.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle  # noqa: E402


def unit_element():
    C = np.eye(64)
    X = np.array([[i / 3.0, j / 3.0, k / 3.0] for k in range(4) for j in range(4) for i in range(4)])
    return C, X


def curved(X):
    Y = X.copy()
    Y[:, 0] += 0.08 * X[:, 0] * X[:, 1]
    Y[:, 1] += 0.05 * X[:, 1] * X[:, 2]
    return Y


def state():
    return np.array([[0.1 + 0.001 * a, -0.02, 0.03, 0.04 - 0.0002 * a] for a in range(64)])


def previous():
    return np.array([[0.04 - 0.0007 * a, -0.01 + 0.0003 * a, 0.015 - 0.0002 * a, 0.0] for a in range(64)])


CASES = {
    "unit_steady": (False, 1.0, 0.17, 0.0),
    "curved_steady": (True, 1.0, 0.17, 0.0),
    "unit_transient": (False, 2.5, 0.17, 0.2),
    "curved_transient": (True, 2.5, 0.17, 0.2),
}


def main():
    out = {}
    C, X = unit_element()
    for name, (is_curved, rho, mu, dt) in CASES.items():
        XX = curved(X) if is_curved else X
        negres, jac = oracle.ns_element(C, XX, state(), previous() if dt > 0 else None, rho, mu, dt,
                                        use_ref=True)
        out[name + "_negres"] = negres
        out[name + "_jac_rows"] = jac[::16].copy()
    np.savez_compressed(Path(__file__).with_name("element_golden.npz"), **out)


if __name__ == "__main__":
    main()
