"""Python mirror of the reference's host interface over the C ABI.

Class and method names follow ModelG/ModelA.h, Stepper.h and measurer.h so a
driver written against the reference reads the same:

    data = ModelAData(json.load(open("input.json")))
    model = ModelA(data)               # lattice on the current CUDA device
    model.initialize()                 # zero start (ModelA.h:408-461)
    step = PV2HBSplit(model, (2, 3))   # evolverType "PV2HBSplit23"
    meas = Measurer(model)
    meas.measure(); step.step(data.atime.dt())

All work runs in liblgv.so; this module only moves parameters and host arrays.
"""
import ctypes as C

import numpy as np

from . import _lib as L


class ModelATime:
    """ModelATime (ModelA.h:32-68)."""

    def __init__(self):
        self.finaltime, self.initialtime, self.deltat, self.time = 10.0, 0.0, 0.24, 0.0

    def t(self): return self.time
    def dt(self): return self.deltat
    def tinitial(self): return self.initialtime
    def tfinal(self): return self.finaltime
    def reset(self): self.time = self.initialtime

    def __iadd__(self, d):
        self.time += d
        return self

    def adjust_finaltime(self, saveFrequency):
        # ModelA.h:48-53: whole number of saveFrequency*dt units
        self.finaltime = self.initialtime + self.deltat * saveFrequency * int(
            (self.finaltime - self.initialtime) / (self.deltat * saveFrequency))
        return self.finaltime

    def read(self, p):
        self.finaltime = float(p.get("finaltime", self.finaltime))
        self.initialtime = float(p.get("initialtime", self.initialtime))
        self.deltat = float(p.get("deltat", self.deltat))
        self.time = self.initialtime


class ModelACoefficients:
    """ModelACoefficients (ModelA.h:71-111)."""

    def __init__(self):
        self.mass0, self.dmassdt, self.lambda_, self.H, self.chi = -4.70052, 0.0, 4.0, 0.003, 5.0
        self.gamma, self.diffusion = 1.0, 0.3333333

    def mass(self, t): return self.mass0 + self.dmassdt * t
    def sigma(self): return self.diffusion * self.chi
    def D(self): return self.diffusion

    def read(self, p):
        self.mass0 = float(p.get("mass0", self.mass0))
        self.dmassdt = float(p.get("dmassdt", 0.0))
        self.lambda_ = float(p.get("lambda", self.lambda_))
        self.H = float(p.get("H", self.H))
        self.chi = float(p.get("chi", self.chi))
        self.gamma = float(p.get("gamma", self.gamma))
        self.diffusion = float(p.get("diffusion", 1.0 / 3.0 * self.gamma))


class ModelAHandlerData:
    """ModelAHandlerData (ModelA.h:114-181)."""

    def __init__(self):
        self.evolverType, self.seed, self.restart = "PV2HBSplit23", 10, False
        self.outputfiletag, self.saveFrequency, self.writeFrequency = "o4output", 3, -1
        self.eventmode, self.nevents, self.current_event = False, 1, 0
        self.thermalization_time, self.quench_mode, self.quench_mode_mass0 = 0.0, False, -4.70052

    def read(self, p):
        self.evolverType = str(p.get("evolverType", self.evolverType))
        self.seed = int(p.get("seed", self.seed))
        self.restart = bool(p.get("restart", False))
        self.outputfiletag = str(p.get("outputfiletag", "o4output"))
        self.saveFrequency = int(p.get("saveFrequency", self.saveFrequency))
        self.writeFrequency = int(p.get("writeFrequency", self.writeFrequency))
        self.thermalization_time = float(p.get("thermalization_time", self.thermalization_time))
        self.quench_mode = bool(p.get("quench_mode", self.quench_mode))
        self.quench_mode_mass0 = float(p.get("quench_mode_mass0", self.quench_mode_mass0))
        self.eventmode = bool(p.get("eventmode", self.eventmode))
        self.nevents = int(p.get("nevents", self.nevents))


class ModelAData:
    """ModelAData (ModelA.h:185-269): the JSON keys of the reference input file."""
    Nphi, NA, NV, Ndof = 4, 3, 3, 10

    def __init__(self, params):
        self.NX = int(params["NX"])
        self.NY = self.NZ = self.NX
        self.LX = float(int(params.get("LX", self.NX)))
        self.LY = self.LZ = self.LX
        self.atime = ModelATime()
        self.acoefficients = ModelACoefficients()
        self.ahandler = ModelAHandlerData()
        self.atime.read(params)
        self.acoefficients.read(params)
        self.ahandler.read(params)
        params["finaltime"] = self.atime.adjust_finaltime(self.ahandler.saveFrequency)

    def hX(self): return self.LX / self.NX
    def mass(self): return self.acoefficients.mass(self.atime.t())

    def lgv_params(self):
        c = self.acoefficients
        return L.make_params(self.NX, LX=self.LX, mass0=c.mass0, dmassdt=c.dmassdt, lam=c.lambda_, H=c.H,
                             chi=c.chi, gamma=c.gamma, diffusion=c.diffusion, seed=self.ahandler.seed)


class ModelA:
    """ModelA (ModelA.h:291-526): owns the device lattice through an lgv handle."""

    def __init__(self, data):
        self.lib = L.load()
        self.data = data
        self.N = data.NX
        self.V = self.N ** 3
        self._params = data.lgv_params()
        h = C.c_void_p()
        L.check(self.lib.lgv_create(C.byref(self._params), C.byref(h)), "lgv_create")
        self.handle = h

    def sync_params(self):
        self._params = self.data.lgv_params()
        L.check(self.lib.lgv_set_params(self.handle, C.byref(self._params)), "lgv_set_params")

    def initialize(self):
        L.check(self.lib.lgv_initialize(self.handle, L.INIT_ZERO, 0.0), "lgv_initialize")

    def initialize_gaussian_phi(self, scale):
        L.check(self.lib.lgv_initialize(self.handle, L.INIT_PHI_GAUSSIAN, float(scale)), "lgv_initialize")

    def initialize_gaussian_charges(self):
        L.check(self.lib.lgv_initialize(self.handle, L.INIT_CHARGES_GAUSSIAN, 0.0), "lgv_initialize")

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == self.V * 10
        L.check(self.lib.lgv_set_state(self.handle, L.ptr(u)), "lgv_set_state")

    def get_state(self):
        u = np.empty((self.N, self.N, self.N, 10))
        L.check(self.lib.lgv_get_state(self.handle, L.ptr(u)), "lgv_get_state")
        return u

    def set_counter(self, c):
        L.check(self.lib.lgv_set_counter(self.handle, int(c)), "lgv_set_counter")

    def set_hb_proposal(self, gaussian):
        """Gaussian phi heat-bath proposals (True) or the reference's uniform
        U(-sqrt3, sqrt3) ones (False, the default); lgv_set_hb_proposal."""
        kind = L.HB_PROPOSAL_GAUSSIAN if gaussian else L.HB_PROPOSAL_UNIFORM
        L.check(self.lib.lgv_set_hb_proposal(self.handle, kind), "lgv_set_hb_proposal")

    def get_counter(self):
        c = C.c_uint64()
        L.check(self.lib.lgv_get_counter(self.handle, C.byref(c)), "lgv_get_counter")
        return c.value

    def diff_forward(self, dt, nsteps, avg_begin, ckpt_every, t=0.0, evolver=L.MODELA_EM):
        """Differentiable run (lgv_diff_forward): returns the time averages
        (sigma, V sum_a pibar_a^2) over steps avg_begin+1 .. nsteps."""
        obs = np.zeros(2)
        L.check(self.lib.lgv_diff_forward(self.handle, int(evolver), float(dt), float(t), int(nsteps), int(avg_begin),
                                          int(ckpt_every), L.ptr(obs)), "lgv_diff_forward")
        return obs

    def diff_backward(self, w=(1.0, 1.0)):
        """Gradient of w[0] obs[0] + w[1] obs[1] of the last diff_forward with respect to
        (mass0, lambda, H, gamma), by the adjoint kernels (lgv_diff_backward)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        g = np.zeros(4)
        L.check(self.lib.lgv_diff_backward(self.handle, L.ptr(w), L.ptr(g)), "lgv_diff_backward")
        return g

    def diff_averages(self, nsteps):
        """Volume averages <phi_a>(n), n = 0..nsteps, of the last diff_forward, shape (nsteps+1, 4)."""
        out = np.zeros((int(nsteps) + 1, 4))
        L.check(self.lib.lgv_diff_averages(self.handle, L.ptr(out), int(nsteps)), "lgv_diff_averages")
        return out

    def energy(self):
        e = C.c_double()
        L.check(self.lib.lgv_energy(self.handle, C.byref(e)), "lgv_energy")
        return e.value

    def synchronize(self):
        L.check(self.lib.lgv_synchronize(self.handle), "lgv_synchronize")

    def finalize(self):
        if getattr(self, "handle", None):
            self.lib.lgv_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass


class Stepper:
    """Stepper (Stepper.h:6-11): step(dt) advances model.data.atime's state."""
    evolver = None

    def __init__(self, model):
        self.model = model

    def _run(self, dt, inner=1, outer=1, nsteps=1, t=None):
        m = self.model
        t = m.data.atime.t() if t is None else t
        L.check(m.lib.lgv_step(m.handle, self.evolver, inner, outer, float(dt), float(t), int(nsteps)),
                "lgv_step")
        return True

    def step(self, dt):
        return self._run(dt)

    def finalize(self):
        pass


class IdealPV2(Stepper):
    evolver = L.IDEAL_PV2


class EulerLangevinHB(Stepper):
    evolver = L.EULER_LANGEVIN_HB


class ModelGChargeHB(Stepper):
    evolver = L.CHARGE_HB


class ModelAEulerMaruyama(Stepper):
    evolver = L.MODELA_EM


class IdealEulerMaruyama(Stepper):
    """Ideal step then Euler-Maruyama relaxation of phi (no counterpart in the reference)."""
    evolver = L.IDEAL_EM


class PV2HBSplit(Stepper):
    """PV2HBSplit (Stepper.h:176-211): scounts = (inner, outer)."""

    def __init__(self, model, scounts=(1, 1), nodiffuse=False, onlydiffuse=False):
        super().__init__(model)
        self.scounts = tuple(scounts)
        self.evolver = (L.PV2HBSPLIT_ONLYDIFFUSE if onlydiffuse else
                        L.PV2HBSPLIT_NODIFFUSE if nodiffuse else L.PV2HBSPLIT)

    def step(self, dt):
        return self._run(dt, self.scounts[0], self.scounts[1])


def make_stepper(model, evolverType):
    """The evolverType switch of SuperPions.cxx:209-225."""
    if evolverType == "PV2HBSplit23":
        return PV2HBSplit(model, (2, 3))
    if evolverType == "PV2HBSplit23NoDiffuse":
        return PV2HBSplit(model, (2, 3), nodiffuse=True)
    if evolverType == "PV2HBSplit23OnlyDiffuse":
        return PV2HBSplit(model, (2, 3), onlydiffuse=True)
    if evolverType == "PV2HBSplit11":
        return PV2HBSplit(model, (1, 1))
    if evolverType == "ModelAEulerMaruyama":
        return ModelAEulerMaruyama(model)
    if evolverType == "IdealEulerMaruyama":
        return IdealEulerMaruyama(model)
    if evolverType == "EulerLangevinHB":
        return EulerLangevinHB(model)
    raise ValueError(f"Unrecognized stepper type {evolverType}")


class Measurer:
    """Measurer (measurer.h:88-194): measure() fills the public arrays."""

    def __init__(self, model):
        self.model = model
        self.N = model.N
        self.result = L.Measurement(self.N)

    def measure(self):
        m = self.model
        s = self.result.struct()
        L.check(m.lib.lgv_measure(m.handle, C.byref(s)), "lgv_measure")
        r = self.result
        self.OAverage = r.OAverage
        for a, ax in enumerate("XYZ"):
            setattr(self, f"wall{ax}", r.wall[a])
            setattr(self, f"wall{ax}_k", r.wall_k[a][..., 0] + 1j * r.wall_k[a][..., 1])
            setattr(self, f"wall{ax}_k_rotated", r.wall_k_rotated[a][..., 0] + 1j * r.wall_k_rotated[a][..., 1])
            setattr(self, f"wall{ax}Phase", r.wall_phase[a])
            setattr(self, f"wall{ax}Phase_k", r.wall_phase_k[a][..., 0] + 1j * r.wall_phase_k[a][..., 1])
        return r
