"""Integrators (gamdpy/integrators/NVE.py, NVT.py, NVT_Langevin.py,
NPT_Atomic.py).

The step itself runs fused with the force evaluation in libgamdb200's step
kernel; these classes carry the parameters with gamdpy's names and
conventions and hand them to the library.
"""
import numpy as np

from . import _lib
from .misc import make_function_constant


class Integrator:
    """Abstract integrator (gamdpy/integrators/integrator.py:4-23)."""


class NVE(Integrator):
    """Leapfrog, total-energy conserving (integrators/NVE.py:8-113):
    v(t+dt/2) = v(t-dt/2) + f(t) dt / m,  r(t+dt) = r(t) + v(t+dt/2) dt."""

    def __init__(self, dt):
        self.dt = dt

    def get_params(self, configuration=None, interactions_params=None, verbose=False):
        return (np.float32(self.dt),)

    def configure_device(self, sim, configuration):
        sim.set_nve(np.float32(self.dt))


class _DeviceState:
    """Stand-in for the reference's ``d_thermostat_state`` device array:
    ``copy_to_host()`` reads the state from the library."""

    def __init__(self, owner):
        self._owner = owner

    def copy_to_host(self):
        return self._owner.thermostat_state.copy() if self._owner._device is None \
            else self._owner._device.thermostat_state()


class NVT(Integrator):
    """Leapfrog with a Nose-Hoover thermostat (integrators/NVT.py:8-141).
    ``temperature`` is a number or a function of time made by
    make_function_constant / make_function_ramp."""

    def __init__(self, temperature, tau, dt):
        self.temperature = temperature
        self.tau = tau
        self.dt = dt
        self.thermostat_state = np.zeros(2, dtype=np.float32)
        self._device = None
        self.d_thermostat_state = _DeviceState(self)

    def get_params(self, configuration, interactions_params=None, verbose=False):
        dt = np.float32(self.dt)
        omega2 = np.float32(4.0 * np.pi * np.pi / self.tau / self.tau)
        degrees = configuration.N * configuration.D - configuration.D
        return (dt, omega2, degrees, self.d_thermostat_state)

    def _tfunc(self):
        T = self.temperature
        if not callable(T):
            T = make_function_constant(value=float(T))
        kind = getattr(T, "_gdb_tfunc", None)
        if kind is None:
            raise NotImplementedError("NVT temperature must be a number, make_function_constant or "
                                      "make_function_ramp (the step runs in CUDA)")
        return kind, T._gdb_tparams

    def configure_device(self, sim, configuration):
        kind, tparams = self._tfunc()
        sim.set_nvt(np.float32(self.dt), float(self.tau), kind, tparams)
        sim.set_thermostat_state(self.thermostat_state)
        self._device = sim

    def sync_from_device(self):
        if self._device is not None:
            self.thermostat_state[:] = self._device.thermostat_state()


class NVT_Langevin(Integrator):
    """Leap-frog Langevin thermostat (integrators/NVT_Langevin.py:12-138;
    Gronbech-Jensen and Farago, arXiv:1303.7011, Eq. 16):
    m a = f - alpha v + beta, with beta = sqrt(2 alpha T dt) times a normal
    number from a per-particle xoroshiro128+ generator seeded as
    numba.cuda.random.create_xoroshiro128p_states(N, seed).  ``temperature``
    is a number or a function of time from make_function_constant /
    make_function_ramp.  Runs on the persistent and graph paths; systems with
    it are not batched."""

    def __init__(self, temperature, alpha: float, dt: float, seed: int) -> None:
        self.temperature = temperature
        self.alpha = alpha
        self.dt = dt
        self.seed = seed

    def get_params(self, configuration, interactions_params=None, verbose=False):
        return (np.float32(self.dt), np.float32(self.alpha), self.seed)

    def _tfunc(self):
        T = self.temperature
        if not callable(T):
            T = make_function_constant(value=float(T))
        kind = getattr(T, "_gdb_tfunc", None)
        if kind is None:
            raise NotImplementedError("NVT_Langevin temperature must be a number, make_function_constant or "
                                      "make_function_ramp (the step runs in CUDA)")
        return kind, T._gdb_tparams

    def configure_device(self, sim, configuration):
        kind, tparams = self._tfunc()
        sim.set_langevin(np.float32(self.dt), np.float32(self.alpha), int(self.seed), kind, tparams)


class NPT_Atomic(Integrator):
    """Constant N, P, T for atomic systems (integrators/NPT_Atomic.py:9-213):
    leap-frog with the Martyna-Tobias-Klein thermostat and barostat
    (Mol. Phys. 87, 1117 (1996)).  ``thermostat_state`` = (p_xi/Q, 0) and
    ``barostat_state`` = (p_eps/W, 0, volume), float32 as in the reference
    (the second entries are the reference's accumulators, zero between
    steps).  ``temperature`` and ``pressure`` are numbers or functions of
    time from make_function_constant / make_function_ramp.  The step, the box
    scaling and the state update run fused in the persistent kernel; the box
    lengths of the configuration follow the run."""

    def __init__(self, temperature, tau: float, pressure, tau_p: float, dt: float) -> None:
        self.temperature = temperature
        self.tau = tau
        self.pressure = pressure
        self.tau_p = tau_p
        self.dt = dt
        self.thermostat_state = np.zeros(2, dtype=np.float32)
        self.barostat_state = np.zeros(3, dtype=np.float32)
        self._device = None

    def _masses(self, configuration):
        # NPT_Atomic.py:43-48 (numpy float32 arithmetic)
        degrees = configuration.N * configuration.D - configuration.D
        factor = np.float32(1. / (4 * np.pi * np.pi))
        mass_t = np.float32((degrees - 1) * configuration.D * factor * self.tau * self.tau)
        mass_p = np.float32((degrees - 1) * configuration.D * factor * self.tau_p * self.tau_p)
        return degrees, mass_t, mass_p

    def get_params(self, configuration, interactions_params=None, verbose=False):
        degrees, mass_t, mass_p = self._masses(configuration)
        self.barostat_state[2] = configuration.get_volume()
        return (np.float32(self.dt), mass_t, mass_p, degrees, self.thermostat_state, self.barostat_state)

    @staticmethod
    def _func(f, what):
        if not callable(f):
            f = make_function_constant(value=float(f))
        kind = getattr(f, "_gdb_tfunc", None)
        if kind is None:
            raise NotImplementedError(f"NPT_Atomic {what} must be a number, make_function_constant or "
                                      "make_function_ramp (the step runs in CUDA)")
        return kind, f._gdb_tparams

    def configure_device(self, sim, configuration):
        _, mass_t, mass_p = self._masses(configuration)
        tk, tp = self._func(self.temperature, "temperature")
        pk, pp = self._func(self.pressure, "pressure")
        sim.set_npt(np.float32(self.dt), mass_t, mass_p, tk, tp, pk, pp)
        self.barostat_state[2] = configuration.get_volume()
        sim.set_npt_state(self.thermostat_state, self.barostat_state)
        self._device = sim

    def sync_from_device(self):
        if self._device is not None:
            ts, bs = self._device.npt_state()
            self.thermostat_state[:] = ts
            self.barostat_state[:] = bs
