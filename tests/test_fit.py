"""The material fitter's parameter update (rfdem.fit.FitTask) against the reference's own
mp_task_data compiled from mp_task.h (oracle reference build): the same result rows give
the same parameters and variations, bit for bit, over several conjugate-gradient steps,
including the clamps and the source's index behaviours."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from rfdem import fit

REF_IO = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libmdref_io.so")


def _reference(nsteps, goal, start, factor, rfunc):
    L = C.CDLL(REF_IO)
    P = C.c_void_p
    L.ref_fit.argtypes = [C.c_int, P, P, C.c_double, P, P, P]
    params = np.zeros((nsteps + 1) * 5)
    var = np.zeros((nsteps + 1) * 30)
    assert L.ref_fit(nsteps, goal.ctypes.data, start.ctypes.data, factor, rfunc.ctypes.data, params.ctypes.data,
                     var.ctypes.data) == 0
    return params.reshape(nsteps + 1, 5), var.reshape(nsteps + 1, 30)


@pytest.mark.skipif(not os.path.exists(REF_IO), reason="reference build absent (oracle/build.py)")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cg_update_matches_reference(seed):
    rng = np.random.default_rng(seed)
    nsteps = 6
    goal, start = fit.granite_goal(), fit.granite_start()
    # result rows near the goal: a base row and five varied rows per step
    rfunc = (goal[None, None, :] * (1.0 + 0.2 * rng.normal(size=(nsteps, 6, 3)))).reshape(nsteps, 18)
    ref_params, ref_var = _reference(nsteps, goal, start, 0.05, np.ascontiguousarray(rfunc))
    T = fit.FitTask(nsteps + 1, goal=goal, start=start)
    T.calculate_start_parameters()
    assert np.array_equal(T.ParameterVariation, ref_var[0])
    for s in range(nsteps):
        T.Step = s
        T.RFunction[:] = rfunc[s]
        T.calculate_new_parameters2()
        assert np.array_equal(T.ParameterVariation, ref_var[s + 1]), s
    got = T.MaterialParametersSteps.reshape(nsteps + 1, 5)
    assert np.array_equal(got.view(np.uint64), ref_params.view(np.uint64)), np.abs(got - ref_params).max()


def test_contractions_and_variations():
    """SetMaterialContractions' clamps, and the variation rows a step runs."""
    T = fit.FitTask(3)
    T.calculate_start_parameters()
    assert all(T.varied(i) for i in range(6))
    p = T.variation(2)                      # run 2 varies Ec by 5 %
    base = T.params()
    assert p[1] == base[1] + 0.05 * base[1] and np.array_equal(np.delete(p, 1), np.delete(base, 1))
    T.MaterialParametersSteps[5:10] = [1e-9, 0.9e-9, 0.0, 0.0, 0.0]
    T.set_material_contractions()
    m = T.MaterialParametersSteps[5:10]
    assert m[0] == 1e+5 / fit.STRESS_CONST and m[1] == 1.4 * m[0]
    assert m[2] == 1e+8 / fit.STRESS_CONST and m[3] == 1e-6 / fit.LENGTH_CONST and m[4] == 1e-5 / fit.LENGTH_CONST
