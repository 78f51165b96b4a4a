// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own conjugate-gradient parameter update, mp_task_data from
// mp_task.h (CalculateStartParameters, CalculateNewParameters2, SetMaterialContractions),
// compiled unmodified into oracle/_ref/libmdref_io.so, on given result rows: the tests
// compare the engine package's restatement (rfdem.fit.FitTask) with it bit for bit. The
// update prints its intermediate values to std::cerr; the stream is muted for the call.

#include <cstring>
#include <iostream>
#include "mp_task.h"

extern "C" {

// nsteps updates; rfunc: nsteps x (NResult * (NParam + 1)) result rows; outputs the
// parameters of steps 0..nsteps ((nsteps + 1) x NParam) and the variation table after
// the start and after each update ((nsteps + 1) x (NParam + 1) x NParam).
int ref_fit(int nsteps, const double* goal, const double* start, double factor, const double* rfunc,
            double* params_out, double* variation_out) {
    mp_task_data T;
    T.NSteps = (uint_fast32_t)nsteps + 1;
    T.NParam = 5;
    T.NResult = 3;
    T.MaterialDeltaFactor = factor;
    T.createarrays();
    const size_t np = T.NParam, nr = T.NResult, nv = (np + 1) * np, nrf = nr * (np + 1);
    for (size_t j = 0; j < nr; ++j) T.ResultsGoal[j] = goal[j];
    for (size_t i = 0; i < np; ++i) T.MaterialParametersSteps[i] = start[i];
    T.Step = 0;
    T.CalculateStartParameters();
    std::memcpy(variation_out, T.ParameterVariation, nv * sizeof(double));
    std::streambuf* saved = std::cerr.rdbuf(nullptr);
    for (int s = 0; s < nsteps; ++s) {
        T.Step = (uint_fast32_t)s;
        std::memcpy(T.RFunction, rfunc + (size_t)s * nrf, nrf * sizeof(double));
        T.CalculateNewParameters2();
        std::memcpy(variation_out + (size_t)(s + 1) * nv, T.ParameterVariation, nv * sizeof(double));
    }
    std::cerr.rdbuf(saved);
    std::cerr.clear();
    std::memcpy(params_out, T.MaterialParametersSteps, (size_t)(nsteps + 1) * np * sizeof(double));
    return 0;
}

}  // extern "C"
