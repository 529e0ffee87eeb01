"""Host logic of the Python mirror on the CPU (no GPU call): ModelAData reads
the reference's JSON keys with its defaults and quirks (ModelA.h:32-269),
maps onto lgv_params, and the evolverType switch and stepper classes are
those of SuperPions.cxx:209-225 / Stepper.cxx:537-580."""
import math

import pytest


def data(**kw):
    from langevina_b200 import ModelAData

    return ModelAData(dict(kw))


def test_defaults_and_finaltime_adjustment():
    d = data(NX=16)
    c, t, h = d.acoefficients, d.atime, d.ahandler
    assert (c.mass0, c.dmassdt, c.lambda_, c.H, c.chi, c.gamma) == (-4.70052, 0.0, 4.0, 0.003, 5.0, 1.0)
    # diffusion defaults to gamma / 3 when absent (ModelA.h:98)
    assert c.diffusion == pytest.approx(1.0 / 3.0)
    assert (t.initialtime, t.deltat, t.time) == (0.0, 0.24, 0.0)
    # finaltime = initialtime + dt * saveFrequency * floor((10 - 0) / (0.24 * 3)) (ModelA.h:48-53)
    assert t.finaltime == pytest.approx(0.24 * 3 * 13)
    assert (h.evolverType, h.seed, h.restart, h.outputfiletag) == ("PV2HBSplit23", 10, False, "o4output")
    assert (h.saveFrequency, h.writeFrequency, h.eventmode, h.nevents) == (3, -1, False, 1)
    assert (h.thermalization_time, h.quench_mode, h.quench_mode_mass0) == (0.0, False, -4.70052)
    assert (d.NX, d.NY, d.NZ, d.LX, d.hX()) == (16, 16, 16, 16.0, 1.0)


def test_keys_and_quirks():
    params = {"NX": 8, "LX": 12.7, "gamma": 2.0, "lambda": 10, "mass0": -4.813, "dmassdt": 0.5, "H": 0.01,
              "chi": 3.0, "deltat": 0.04, "finaltime": 1.0, "initialtime": 0.2, "saveFrequency": 10,
              "seed": 77, "evolverType": "PV2HBSplit23NoDiffuse", "quench_mode": True, "quench_mode_mass0": -5.0,
              "eventmode": True, "nevents": 3, "thermalization_time": 2.0, "writeFrequency": 5}
    from langevina_b200 import ModelAData

    d = ModelAData(params)
    c, t, h = d.acoefficients, d.atime, d.ahandler
    assert d.LX == 12.0 and d.hX() == 1.5  # LX is read as an integer (ModelA.h:229)
    assert c.diffusion == pytest.approx(2.0 / 3.0)  # gamma / 3 with the gamma read first
    assert (c.lambda_, c.mass0, c.dmassdt, c.H, c.chi) == (10.0, -4.813, 0.5, 0.01, 3.0)
    assert t.time == 0.2 and t.deltat == 0.04
    n = math.floor((1.0 - 0.2) / (0.04 * 10))
    assert t.finaltime == pytest.approx(0.2 + 0.04 * 10 * n)
    assert params["finaltime"] == t.finaltime  # written back into the input, as the reference does
    assert d.mass() == pytest.approx(-4.813 + 0.5 * 0.2)
    assert (h.seed, h.evolverType, h.quench_mode, h.quench_mode_mass0) == (77, "PV2HBSplit23NoDiffuse", True, -5.0)
    assert (h.eventmode, h.nevents, h.thermalization_time, h.writeFrequency) == (True, 3, 2.0, 5)


def test_lgv_params_mapping():
    d = data(NX=32, LX=64, mass0=-4.813, dmassdt=0.1, H=0.006, chi=5.0, gamma=1.5, diffusion=0.25, seed=123,
             **{"lambda": 10.0})
    p = d.lgv_params()
    assert (p.N, p.reserved0, p.LX, p.mass0, p.dmassdt, p.lambda_, p.H, p.chi, p.gamma, p.diffusion, p.seed) == \
        (32, 0, 64.0, -4.813, 0.1, 10.0, 0.006, 5.0, 1.5, 0.25, 123)


def test_timekeeping():
    d = data(NX=4, deltat=0.1, finaltime=1.0, saveFrequency=1, initialtime=0.5)
    t = d.atime
    t += t.dt()
    t += t.dt()
    assert t.t() == pytest.approx(0.7)
    t.reset()
    assert t.t() == 0.5 and t.tinitial() == 0.5 and t.tfinal() == pytest.approx(1.0)


def test_evolver_names():
    """make_stepper's switch (SuperPions.cxx:209-225 and the extra steppers)
    without a device: the classes and their sub-step counts."""
    from langevina_b200 import _lib as L
    from langevina_b200 import model as M

    class FakeModel:
        pass

    want = {"PV2HBSplit23": (L.PV2HBSPLIT, (2, 3)), "PV2HBSplit23NoDiffuse": (L.PV2HBSPLIT_NODIFFUSE, (2, 3)),
            "PV2HBSplit23OnlyDiffuse": (L.PV2HBSPLIT_ONLYDIFFUSE, (2, 3)), "PV2HBSplit11": (L.PV2HBSPLIT, (1, 1))}
    for name, (ev, sc) in want.items():
        s = M.make_stepper(FakeModel(), name)
        assert isinstance(s, M.PV2HBSplit) and s.evolver == ev and tuple(s.scounts) == sc, name
    assert isinstance(M.make_stepper(FakeModel(), "ModelAEulerMaruyama"), M.ModelAEulerMaruyama)
    assert isinstance(M.make_stepper(FakeModel(), "IdealEulerMaruyama"), M.IdealEulerMaruyama)
    assert isinstance(M.make_stepper(FakeModel(), "EulerLangevinHB"), M.EulerLangevinHB)
    with pytest.raises(ValueError):
        M.make_stepper(FakeModel(), "PV2HBSplit99")
