"""Generates tests/golden/python_fe_truss.json from the reference's own
Python FE restatement (test/python_fe: TrussFE, truss_fe.py; DynamicSolver,
dynamic_solver.py:20-101), run where the reference tree is available; the
JSON is committed so the tests never read the reference.

The solver is configured as the explicit central difference of the path:
alpha = 0, beta = 1/2, unknown = acceleration ('acce'), whose Jacobian is
then the mass matrix alone; the truss model's mass is lumped (row sums of
its consistent mass matrix, the reference's assembleMassLumped for
segment_2: rho A Le / 2 per element end). One step is then predictor,
a = M^-1 (f_ext - K u), corrector: the lumped explicit step.

Cases: a 1D bar of E, rho, length L in Ne segment_2 elements, node 0 fixed
at u = 0, a load on the last node, initial displacement sin(pi x / 2L),
dt = 0.5 Le / c; the displacement of every node after each of the first
steps is stored.

usage: python tests/golden/make_python_fe.py REFERENCE_ROOT
"""
import contextlib
import io
import json
import math
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))

# tolerance: the solver's absolute convergence test on the correction
# (dynamic_solver.py:88-93), scaled to each case's accelerations
CASES = [dict(E=1.0, rho=1.0, L=1.0, Ne=10, F=-0.1, steps=60, tolerance=1e-10),
         dict(E=210e9, rho=7800.0, L=2.0, Ne=25, F=-1e5, steps=80, tolerance=1e-3)]


def main(ref):
    sys.path.insert(0, os.path.join(ref, "test"))
    from python_fe.dynamic_solver import DynamicSolver
    from python_fe.truss_fe import TrussFE

    class LumpedTrussFE(TrussFE):
        def assembleMass(self):
            super().assembleMass()
            self._M = sp.diags(np.asarray(self._M.sum(axis=1)).ravel()).tocsr()

    out = []
    for c in CASES:
        Ne, L = c["Ne"], c["L"]
        model = LumpedTrussFE(A=1.0, E=c["E"], L=L, rho=c["rho"], Ne=Ne,
                              F={c["F"]: [Ne]}, blocked=([0], [0.0]))
        x = np.linspace(0.0, L, Ne + 1)
        model.u = 1e-3 * L * np.sin(math.pi * x / (2 * L))
        dt = 0.5 * (L / Ne) / math.sqrt(c["E"] / c["rho"])
        # the coefficient table (dynamic_solver.py:31-41) divides by alpha for
        # the 'disp' and 'velo' unknowns; build it with alpha = 1, then give
        # the one alpha-dependent coefficient of the 'acce' unknown (its
        # displacement update, alpha beta dt^2) its alpha = 0 value
        solver = DynamicSolver(model, delta_t=dt, alpha=1.0, beta=0.5, type="acce",
                               tolerance=c["tolerance"])
        solver._coeff["acce"]["disp"] = 0.0
        traj = []
        with contextlib.redirect_stdout(io.StringIO()):
            for _ in range(c["steps"]):
                solver.solveStep()
                traj.append(model.u.tolist())
        out.append(dict(c, dt=dt, x=x.tolist(), u0=(1e-3 * L * np.sin(math.pi * x / (2 * L))).tolist(),
                        displacement=traj))
    with open(os.path.join(HERE, "python_fe_truss.json"), "w") as fh:
        json.dump({"source": "test/python_fe (TrussFE, DynamicSolver)", "cases": out}, fh)
    print("wrote", os.path.join(HERE, "python_fe_truss.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
