"""The material fitter on the GPU: the 12 simulations of a conjugate-gradient step run
concurrently (one engine per run, all launched before any is waited on) give exactly the
results of running them one after the other, and the base uniaxial run equals the
drop-in driver md_CalculationUniaxialCompression on the same task."""
import numpy as np
import pytest

import rfdem
from rfdem import fit

pytestmark = pytest.mark.gpu


def test_concurrent_runs_equal_sequential_and_driver(cuda):
    S = fit.Specimens(uni=(6.0, 10.0), brazil=(10.0, 4.0))
    a = fit.FitTask(3)
    a.calculate_start_parameters()
    b = fit.FitTask(3)
    b.calculate_start_parameters()
    sa = fit.evaluate(a, S, max_steps=200_000, concurrent=True)
    sb = fit.evaluate(b, S, max_steps=200_000, concurrent=False)
    assert sa == sb
    assert np.array_equal(a.RFunction, b.RFunction)
    assert np.all(a.RFunction > 0)                          # every run reached a fracture stress
    assert all(n < 200_000 for n in sa.values())            # and stopped at its fracture
    t, R = S.task(rfdem.RF_TEST_UNIAXIAL, a.variation(0))
    res, _, _ = rfdem.run_test(t, R, max_steps=200_000)
    assert res.steps == sa[(0, rfdem.RF_TEST_UNIAXIAL)]
    assert (t.Compress.FractureStrain, t.Compress.FractureStress) == (a.RFunction[0], a.RFunction[1])
    # the update consumes the rows
    p0 = a.params()
    a.calculate_new_parameters2()
    a.Step += 1
    p1 = a.params()
    assert np.all(np.isfinite(p1)) and not np.array_equal(p0, p1)
