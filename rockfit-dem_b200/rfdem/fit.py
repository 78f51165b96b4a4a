"""Material fitting: the reference's conjugate-gradient fitter on the fused engine.

The reference fits five material parameters -- Young's modulus E, the bond tensile and
shear strengths Ec and Gc, the bond radius b_r and the bonding gap (b_d - 2 p_r) -- to
three measured results of granite -- uniaxial fracture strain and strength and the
Brazilian (tensile) strength. Each conjugate-gradient step runs the base parameter set
and one forward-difference variation per parameter, each through both tests: 12
simulations (mp_determineconjgradient.cu:84-124), then updates the parameters
(mp_task.h:211-283, CalculateNewParameters2, with the clamps of SetMaterialContractions,
mp_task.h:91-112).

FitTask restates the reference's update arithmetic operation for operation (double,
same order), including two behaviours of the source kept on purpose:
  * the finite-difference quotient of parameter i and result j divides by the variation
    of parameter j (the source indexes the variation by the result, mp_task.h:222-227);
  * SetMaterialContractions moves Ec to 1.4 E when (E - Ec)/E < 0.4 and to 0.6 E when it
    is above 0.4 (mp_task.h:98-106).
evaluate() runs the 12 simulations of a step as one batch: one reference-model engine
per run, every run launched on its own stream before any is waited on, so they share
the GPU; each engine stops at its own fracture.
"""
import numpy as np

# md_phys_constants.h, evaluated as the reference evaluates them
LENGTH_CONST = 1e-3
MASS_CONST = 1e-6
TIME_CONST = 1e-6
FORCE_CONST = MASS_CONST * LENGTH_CONST / (TIME_CONST * TIME_CONST)
STRESS_CONST = FORCE_CONST / (LENGTH_CONST * LENGTH_CONST)
VELOCITY_CONST = LENGTH_CONST / TIME_CONST

NPARAM, NRESULT = 5, 3
VARFLAGS = ((1, 1, 1, 0, 0), (0, 0, 0, 1, 1), (1, 1, 1, 1, 1))


def granite_goal():
    """ResultsGoal of DetermineConjGradient (mp_determineconjgradient.cu:145-149)."""
    return np.array([0.00480002, 104.0497482e6 / STRESS_CONST, 10.5e6 / STRESS_CONST])


def granite_start():
    """The start parameters (mp_determineconjgradient.cu:150-154): E, Ec, Gc, b_r, gap."""
    return np.array([1.95255e+11 / STRESS_CONST, 5.1447e+08 / STRESS_CONST, 3.7131e+08 / STRESS_CONST,
                     0.5 * 0.000330015 / LENGTH_CONST, 5.93169e-05 / LENGTH_CONST])


class FitTask:
    """mp_task_data (mp_task.h:11-90): parameter history, variations and the CG state."""

    def __init__(self, nsteps, goal=None, start=None, delta_factor=0.05):
        self.NSteps, self.NParam, self.NResult = int(nsteps), NPARAM, NRESULT
        self.Step = 0
        self.MaterialDeltaFactor = float(delta_factor)
        self.MaterialParametersSteps = np.zeros(self.NSteps * NPARAM)
        self.ParameterVariation = np.zeros((NPARAM + 1) * NPARAM)
        self.RFunction = np.zeros(NRESULT * (NPARAM + 1))
        self.dRFunction = np.zeros(NRESULT * (NPARAM + 1))
        self.dFunctional = np.zeros(NPARAM + 1)
        self.ddFunctional = np.zeros(NPARAM + 1)
        self.Functional = np.zeros(NRESULT)
        self.DFunctional = np.zeros(NRESULT)
        self.FunctionalParametersWeight = np.zeros(NRESULT)
        self.ResultsGoal = np.array(granite_goal() if goal is None else goal, np.float64)
        self.MaterialParametersSteps[:NPARAM] = granite_start() if start is None else start

    def params(self, step=None):
        s = self.Step if step is None else step
        return self.MaterialParametersSteps[s * NPARAM:(s + 1) * NPARAM].copy()

    def variation(self, i):
        """Parameters of run i of the current step: the step's set plus variation row i
        (SetVariationParameters, mp_determineconjgradient.cu:47-71)."""
        base = self.Step * NPARAM
        return np.array([self.MaterialParametersSteps[base + q] + self.ParameterVariation[NPARAM * i + q]
                         for q in range(NPARAM)])

    def varied(self, i):
        """False for a run the reference skips (a zero variation row, :69)."""
        pv = self.ParameterVariation
        return i == 0 or not (pv[NPARAM * i + 0] + pv[NPARAM * i + 1] + pv[NPARAM * i + 2] + pv[NPARAM * i + 3] +
                              pv[NPARAM * i + 4] < 1e-12)

    def calculate_start_parameters(self):
        """CalculateStartParameters (mp_task.h:113-127)."""
        self.ParameterVariation[:] = 0.0
        for j in range(NRESULT):
            self.FunctionalParametersWeight[j] = 1.0 / (self.ResultsGoal[j] * self.ResultsGoal[j])
        for i in range(NPARAM):
            self.ParameterVariation[NPARAM * (i + 1) + i] = (VARFLAGS[2][i] * self.MaterialDeltaFactor *
                                                            self.MaterialParametersSteps[self.Step * NPARAM + i])

    def set_material_contractions(self):
        """SetMaterialContractions (mp_task.h:91-112) on the next step's parameters."""
        m = self.MaterialParametersSteps
        b = NPARAM * (self.Step + 1)
        d = 0.4
        if m[b + 0] < 1e+5 / STRESS_CONST:
            m[b + 0] = 1e+5 / STRESS_CONST
        if m[b + 1] < 1e+5 / STRESS_CONST:
            m[b + 1] = 1e+5 / STRESS_CONST
        a = (m[b + 0] - m[b + 1]) / m[b + 0]
        if a < d:
            m[b + 1] = (1.0 + d) * m[b + 0]
        elif a > d:
            m[b + 1] = (1.0 - d) * m[b + 0]
        if m[b + 2] < 1e+8 / STRESS_CONST:
            m[b + 2] = 1e+8 / STRESS_CONST
        if m[b + 3] < 1e-6 / LENGTH_CONST:
            m[b + 3] = 1e-6 / LENGTH_CONST
        if m[b + 4] < 1e-5 / LENGTH_CONST:
            m[b + 4] = 1e-5 / LENGTH_CONST

    def calculate_new_parameters2(self):
        """CalculateNewParameters2 (mp_task.h:211-283): finite-difference sensitivities,
        Fletcher-Reeves direction, exact line step of the quadratic model, clamps, and the
        next step's variations."""
        norm = (1.0, 1.0, 1.0, 1.0, 1.0)
        NP, NR = NPARAM, NRESULT
        RF, dRF, PV = self.RFunction, self.dRFunction, self.ParameterVariation
        W, DF, dF, ddF = self.FunctionalParametersWeight, self.DFunctional, self.dFunctional, self.ddFunctional
        for j in range(NR):
            dRF[j] = 0.0
        for i in range(NP):
            for j in range(NR):
                if PV[NP * (j + 1) + j] > 1e-12:
                    dRF[NR * (i + 1) + j] = norm[i] * (RF[NR * (i + 1) + j] - RF[j]) / PV[NP * (j + 1) + j]
                else:
                    dRF[NR * (i + 1) + j] = 0.0
        for j in range(NR):
            DF[j] = self.ResultsGoal[j] - RF[j]
            self.Functional[j] = W[j] * DF[j] * DF[j]
        dF_0 = 0.0
        dF_1 = 0.0
        for i in range(NP):
            ddF[i + 1] = dF[i + 1]
            dF_0 += dF[i + 1] * dF[i + 1]
            dF[i + 1] = 0.0
            for j in range(NR):
                dF[i + 1] += -2.0 * W[j] * DF[j] * dRF[NR * (i + 1) + j]
            dF_1 += dF[i + 1] * dF[i + 1]
        bcoeff = dF_1 / dF_0 if dF_0 > 1e-12 else 0.0
        for i in range(NP):
            ddF[i + 1] = dF[i + 1] + bcoeff * ddF[i + 1]
        a0 = 0.0
        a1 = 0.0
        for j in range(NR):
            for i in range(NP):
                a1 += W[j] * DF[j] * dRF[NR * (i + 1) + j] * ddF[i + 1]
                for k in range(NP):
                    a0 += W[j] * dRF[NR * (i + 1) + j] * ddF[i + 1] * dRF[NR * (k + 1) + j] * ddF[k + 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            tcoeff = float(np.float64(-a1) / np.float64(a0))       # IEEE quotient, as the source divides
        m = self.MaterialParametersSteps
        for i in range(NP):
            m[(self.Step + 1) * NP + i] = m[self.Step * NP + i] - tcoeff * ddF[i + 1] / norm[i]
        self.set_material_contractions()
        PV[:] = 0.0
        for i in range(NP):
            PV[NP * (i + 1) + i] = VARFLAGS[2][i] * self.MaterialDeltaFactor * m[(self.Step + 1) * NP + i]


def material(params):
    """The reference-model potential of one parameter set (SetVariationParameters,
    mp_determineconjgradient.cu:47-67): E, Ec, Gc, b_r, b_d = 2 p_r + gap; the rest fixed."""
    from . import Potential
    po = Potential()
    po.m_nu = 0.247
    po.m_E, po.m_Ec, po.m_Gc = float(params[0]), float(params[1]), float(params[2])
    po.m_ro = 2610 / (MASS_CONST / (LENGTH_CONST * LENGTH_CONST * LENGTH_CONST))
    po.b_r = float(params[3])
    po.p_r = 0.5 * 0.001 / LENGTH_CONST
    po.b_d = 2.0 * po.p_r + float(params[4])
    po.p_e = 0.6
    po.p_mu = 0.45
    po.p_mur = 0.05
    po.a_farcut = 2.9 * po.p_r
    return po


class Specimens:
    """The two specimens every run uses (the reference loads them from its sample files,
    mp_determineconjgradient.cu:177-178): a lattice cylinder for the uniaxial test and a
    lattice disc for the Brazilian test, built once with the start material."""

    def __init__(self, uni=(12.5, 25.0), brazil=(25.0, 10.0), seed=0xB2000000 + 7000):
        from . import RF_TEST_BRAZIL, RF_TEST_UNIAXIAL
        self.shapes = {RF_TEST_UNIAXIAL: uni, RF_TEST_BRAZIL: brazil}
        self.seed = seed

    def task(self, kind, params):
        """(task, positions) of one run: the specimen prepared with the run's material and
        the reference's loading (-0.2 m/s uniaxial with MinStress 15 MPa, -2 m/s Brazilian
        with 2.1 MPa, MaxStrain 0.1; :98-100, :118-120)."""
        from . import RF_TEST_UNIAXIAL, make_test
        d, h = self.shapes[kind]
        v = (-10.0 if kind == RF_TEST_UNIAXIAL else -100.0) * 0.02 / VELOCITY_CONST
        smin = (15e6 if kind == RF_TEST_UNIAXIAL else 2.1e6) / STRESS_CONST
        return make_test(kind, d, h, seed=self.seed + kind, potential=material(params), v_load=v, min_stress=smin,
                         max_strain=0.1)


def evaluate(fit, specimens, max_steps=2_000_000, concurrent=True):
    """The 12 simulations of the current step (CalculateStepCG, :84-124): RFunction rows
    (uniaxial fracture strain and strength, Brazilian strength) for the base set and each
    variation. concurrent: every engine is launched before any is waited on. Returns the
    per-run step counts."""
    from . import RF_TEST_BRAZIL, RF_TEST_UNIAXIAL, Engine
    runs = []
    for i in range(NPARAM + 1):
        if not fit.varied(i):
            continue
        p = fit.variation(i)
        for kind in (RF_TEST_UNIAXIAL, RF_TEST_BRAZIL):
            t, R = specimens.task(kind, p)
            runs.append((i, kind, Engine(t, R)))
    try:
        if concurrent:
            for _, _, e in runs:
                e.step(max_steps)
        steps = {}
        for i, kind, e in runs:
            if not concurrent:
                e.step(max_steps)
            _, r = e.sync()
            steps[(i, kind)] = int(r.steps)
            if kind == RF_TEST_UNIAXIAL:
                fit.RFunction[NRESULT * i + 0] = r.FractureStrain
                fit.RFunction[NRESULT * i + 1] = r.FractureStress
            else:
                fit.RFunction[NRESULT * i + 2] = r.FractureStress
        for i in range(NPARAM + 1):
            if not fit.varied(i):
                fit.RFunction[NRESULT * i:NRESULT * (i + 1)] = 0.0
        return steps
    finally:
        for _, _, e in runs:
            e.close()


def fit_step(fit, specimens, **kw):
    """One conjugate-gradient step: the 12 runs, then the parameter update."""
    steps = evaluate(fit, specimens, **kw)
    fit.calculate_new_parameters2()
    fit.Step += 1
    return steps
