"""Integrators (gamdpy/integrators/NVE.py, NVT.py, NVT_Langevin.py).

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
