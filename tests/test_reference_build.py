"""The oracle against the reference itself, run here.

oracle/_ref/ref_stepper is the reference's unmodified Stepper.cxx,
NoiseGenerator.cxx, measurer.cxx and jsoncpp.cpp (ModelG/), compiled against
the PETSc/MPI/FFTW stand-ins of oracle/shim/ and driven by
oracle/ref_stepper_main.cpp the way SuperPions.cxx's run_event drives it.  With
the reference's own serial noise (NoiseGenerator.h:62-157) the oracle's
SEQUENTIAL mode must reproduce it bit for bit:

- PV2HBSplit::step with scounts {2,3} and {1,1} (Stepper.cxx:542-580), the
  NoDiffuse / OnlyDiffuse forms, and each sub-stepper alone: IdealPV2
  (Stepper.cxx:23-202, including its statistics draw), EulerLangevinHB
  (:287-389) and ModelGChargeHB (:443-522, including std::shuffle of the pass
  order) -- states equal, accept counts equal;
- ModelA::initialize_gaussian_charges (ModelA.h:463-525);
- Measurer::measure (measurer.cxx:10-317): x-space walls bit for bit; the k
  walls to 1e-14 (the reference build's FFTW stand-in is a long-double direct
  DFT, the oracle's a double one);
- IdealPV2::computeEnergy (Stepper.cxx:204-268);
- several MPI ranks (z-slabs, one serial stream per rank seeded as rank r of
  R): the oracle's rank emulation equals the reference's decomposition.
"""
import numpy as np
import pytest

import oracle
import refbuild

pytestmark = pytest.mark.skipif(not refbuild.available(),
                                reason="oracle/_ref/ref_stepper not built (make -C oracle ref REF=<ModelG dir>)")

COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0)
PV2, NODIFF, ONLYDIFF, IDEAL, HB, CHARGE = 0, 1, 2, 3, 4, 5
MON = {"Phi HB Steps": 1, "Charge HB Steps": 2}


def seeded_state(N, seed):
    rng = np.random.default_rng(seed)
    u = np.zeros((N, N, N, 10))
    u[..., :4] = 0.6 * rng.normal(size=(N, N, N, 4))
    u[..., 4:] = np.sqrt(5.0) * rng.normal(size=(N, N, N, 6))
    return u


def oracle_run(N, seed, u, ev, steps, dt, ranks=1, inner=1, outer=1, coef=COEF):
    o = oracle.Oracle(N, mode=oracle.SEQUENTIAL, nranks=ranks, seed=seed, **coef)
    o.set_state(u)
    o.step(ev, dt, t=0.0, nsteps=steps, inner=inner, outer=outer)
    return o


def compare_stats(res, o):
    for name, which in MON.items():
        if name not in res.stats:
            continue
        m = o.monitor(which)
        got = res.stats[name]
        assert (got["up_yes"], got["up_no"], got["down_counts"]) == (m["up_yes"], m["up_no"], m["down_counts"]), name


def compare_measurement(ref_m, o, N):
    from langevina_b200 import _lib as L
    om = o.measure(L.Measurement(N)).arrays()
    for name, want in ref_m.items():
        got = om[name]
        if name == "OAverage" or (name.startswith("wall") and "_k" not in name):
            assert np.array_equal(got, want), name  # bit for bit
        else:
            assert np.max(np.abs(got - want)) < 1e-14, (name, np.max(np.abs(got - want)))


@pytest.mark.parametrize("N,ranks", [(8, 1), (16, 1), (32, 1), (16, 2), (12, 3)])
@pytest.mark.parametrize("inner,outer", [(2, 3), (1, 1)])
def test_pv2hbsplit_equals_reference(N, ranks, inner, outer):
    seed = 1000 + N + ranks
    u = seeded_state(N, seed)
    dt = 0.04
    steps = 2
    res = refbuild.run(refbuild.params_json(N, seed=seed, dt=dt, **COEF),
                       [f"step=PV2HBSplit{inner}{outer},{steps}", "save", "measure", "finalize"], state=u, ranks=ranks)
    o = oracle_run(N, seed, u, PV2, steps, dt, ranks=ranks, inner=inner, outer=outer)
    assert np.array_equal(res.states[0], o.get_state())
    if ranks == 1:  # the reference prints rank 0's statistics only
        compare_stats(res, o)
    compare_measurement(res.measurements[0], o, N)


@pytest.mark.parametrize("name,ev", [("PV2HBSplit23NoDiffuse", NODIFF), ("PV2HBSplit23OnlyDiffuse", ONLYDIFF),
                                     ("IdealPV2", IDEAL), ("EulerLangevinHB", HB), ("ModelGChargeHB", CHARGE)])
def test_substeppers_equal_reference(name, ev):
    N, seed, dt = 12, 77, 0.05
    u = seeded_state(N, seed)
    res = refbuild.run(refbuild.params_json(N, seed=seed, dt=dt, **COEF), [f"step={name},3", "save", "finalize"],
                       state=u)
    o = oracle_run(N, seed, u, ev, 3, dt, inner=2, outer=3)
    assert np.array_equal(res.states[0], o.get_state())
    compare_stats(res, o)
    assert res.stats or ev == IDEAL


def test_time_dependent_mass_equals_reference():
    """m^2(t) = mass0 + dmassdt t (ModelA.h:84) with the clock of run_event."""
    N, seed, dt = 8, 5, 0.04
    coef = dict(COEF, dmassdt=3.0)
    u = seeded_state(N, seed)
    res = refbuild.run(refbuild.params_json(N, seed=seed, dt=dt, **coef), ["step=PV2HBSplit23,4", "save"], state=u)
    o = oracle_run(N, seed, u, PV2, 4, dt, inner=2, outer=3, coef=coef)
    assert np.array_equal(res.states[0], o.get_state())


@pytest.mark.parametrize("ranks", [1, 2])
def test_gaussian_charges_equal_reference(ranks):
    N, seed = 10, 31
    u = seeded_state(N, seed)
    res = refbuild.run(refbuild.params_json(N, seed=seed, **COEF), ["charges", "save"], state=u, ranks=ranks)
    o = oracle.Oracle(N, mode=oracle.SEQUENTIAL, nranks=ranks, seed=seed, **COEF)
    o.set_state(u)
    o.initialize(2)  # LGV_INIT_CHARGES_GAUSSIAN
    assert np.array_equal(res.states[0], o.get_state())


def test_energy_equals_reference():
    N, seed = 10, 9
    u = seeded_state(N, seed)
    res = refbuild.run(refbuild.params_json(N, seed=seed, **COEF), ["energy"], state=u)
    o = oracle.Oracle(N, mode=oracle.SEQUENTIAL, seed=seed, **COEF)
    o.set_state(u)
    assert res.energies[0] == o.energy()


def test_measurer_zero_field_equals_reference():
    """sigma^2 below 100 DBL_MIN takes n = (1,0,0,0) (measurer.cxx:153-159)."""
    N = 8
    u = seeded_state(N, 3)
    u[:, :, ::2, :4] = 0.0
    res = refbuild.run(refbuild.params_json(N, seed=3, **COEF), ["measure"], state=u)
    o = oracle.Oracle(N, mode=oracle.SEQUENTIAL, seed=3, **COEF)
    o.set_state(u)
    compare_measurement(res.measurements[0], o, N)


def test_thermalisation_loop_equals_reference():
    """thermalize_event's inner loop: EulerLangevinHB.step(dt / 6), clock held (SuperPions.cxx:47-53)."""
    N, seed, dt = 8, 12, 0.04
    u = seeded_state(N, seed)
    res = refbuild.run(refbuild.params_json(N, seed=seed, dt=dt, **COEF), ["sub=EulerLangevinHB,12,6", "save"], state=u)
    o = oracle_run(N, seed, u, HB, 12, dt / 6)
    assert np.array_equal(res.states[0], o.get_state())
