"""Runtime actions (gamdpy/runtime_actions/): actions inside the step loop.

ScalarSaver, MomentumReset and ConfigurationSaver keep gamdpy's constructors,
validation and output layout; their per-step work runs inside the library's
step kernel (float64 sums reduced in a fixed order), the host side only
configures it and copies results out at the end of each timeblock.
"""
import math

import numpy as np


class RuntimeAction:
    """Abstract runtime action (gamdpy/runtime_actions/runtime_action.py:7-56)."""

    def get_compute_flags(self):
        return None

    def setup(self, configuration, num_timeblocks, steps_per_timeblock, output, verbose=False):
        pass

    def update_at_end_of_timeblock(self, timeblock, output):
        pass

    def initialize_before_timeblock(self):
        pass


def _check_nonneg_int(name, value):
    if type(value) != int or value < 0:
        raise ValueError(f"{name} ({value}) should be non-negative integer.")


class ScalarSaver(RuntimeAction):
    """Sums of per-particle scalars every ``steps_between_output`` steps
    (runtime_actions/scalar_saver.py:9-206).  Output dataset
    ``scalars[block, save, column]`` float32 with attrs ``scalar_names`` and
    ``steps_between_output`` (scalar_saver.py:172-179)."""

    def __init__(self, steps_between_output: int = 16, compute_flags=None, verbose=False):
        if type(steps_between_output) != int or steps_between_output < 0:
            raise ValueError(f"steps_between_output ({steps_between_output}) should be non-negative integer.")
        self.steps_between_output = steps_between_output
        self.compute_flags = compute_flags

    def get_compute_flags(self):
        return self.compute_flags

    def setup(self, configuration, num_timeblocks, steps_per_timeblock, output, verbose=False):
        self.configuration = configuration
        _check_nonneg_int("num_timeblocks", num_timeblocks)
        _check_nonneg_int("steps_per_timeblock", steps_per_timeblock)
        self.num_timeblocks = num_timeblocks
        self.steps_per_timeblock = steps_per_timeblock
        if self.steps_between_output >= steps_per_timeblock:
            raise ValueError(f"scalar_output ({self.steps_between_output}) must be less than steps_per_timeblock "
                             f"({steps_per_timeblock})")
        flags = configuration.compute_flags
        if flags["Ptot"] or flags["stresses"]:
            raise NotImplementedError("ScalarSaver Ptot/stress columns are outside the B200 hot path")
        self.sid = {}
        for item in ["U", "W", "lapU", "K", "Fsq", "Vol"]:
            if flags[item]:
                self.sid[item] = len(self.sid)
        self.num_scalars = len(self.sid)
        self.scalar_saves_per_block = self.steps_per_timeblock // self.steps_between_output
        output.create_dataset("scalars", shape=(num_timeblocks, self.scalar_saves_per_block, self.num_scalars),
                              dtype=np.float32)
        output.attrs["steps_between_output"] = self.steps_between_output
        output.attrs["scalar_names"] = list(self.sid.keys())

    def update_from_rows(self, block, rows, output, volume, compute_flags=None):
        """rows: (saves, 6) float64 from the library (U, W, lapU, K, Fsq,
        Vol).  The Vol column is the box volume after each saved step when
        the box changes (NPT_Atomic), zero otherwise, where ``volume`` is
        used.  A column whose compute flag the run leaves off stays zero, as
        the reference's saver sums per-particle values its kernels never
        filled (scalar_saver.py:120-130)."""
        col = {"U": 0, "W": 1, "lapU": 2, "K": 3, "Fsq": 4}
        out = np.zeros((self.scalar_saves_per_block, self.num_scalars), np.float32)
        vol_rows = rows[: self.scalar_saves_per_block, 5]
        for name, idx in self.sid.items():
            if name == "Vol":
                out[:, idx] = vol_rows if np.all(vol_rows > 0) else volume
            elif compute_flags is None or compute_flags.get(name, False):
                out[:, idx] = rows[: self.scalar_saves_per_block, col[name]]
        output["scalars"][block, :] = out


class MomentumReset(RuntimeAction):
    """Zero the total momentum every ``steps_between_reset`` steps
    (runtime_actions/momentum_reset.py:12-103)."""

    def __init__(self, steps_between_reset: int):
        if type(steps_between_reset) != int or steps_between_reset < 0:
            raise ValueError(f"steps_between_momentum_reset ({steps_between_reset}) should be non-negative integer.")
        self.steps_between_reset = steps_between_reset


class ConfigurationSaver(RuntimeAction):
    """Log-spaced positions and images per timeblock
    (runtime_actions/configuration_saver.py:9-141): dataset
    ``block[block, save, {r, r_im}, N, D]`` float32, attr ``vectors_names``;
    with ``include_simbox`` also ``sim_box[block, save, D]``, the box lengths
    at each saved step."""

    def __init__(self, include_simbox=False, verbose=False):
        self.include_simbox = include_simbox
        self.num_vectors = 2
        self.sid = {"r": 0, "r_im": 1}

    def setup(self, configuration, num_timeblocks, steps_per_timeblock, output, verbose=False):
        _check_nonneg_int("num_timeblocks", num_timeblocks)
        _check_nonneg_int("steps_per_timeblock", steps_per_timeblock)
        self.configuration = configuration
        self.num_timeblocks = num_timeblocks
        self.steps_per_timeblock = steps_per_timeblock
        self.conf_per_block = int(math.log2(steps_per_timeblock)) + 2
        output.create_dataset("block", shape=(num_timeblocks, self.conf_per_block, self.num_vectors,
                                              configuration.N, configuration.D), dtype=np.float32)
        output.attrs["vectors_names"] = list(self.sid.keys())
        if self.include_simbox:
            output.create_dataset("sim_box", shape=(num_timeblocks, self.conf_per_block, configuration.D),
                                  dtype=np.float32)

    def update_from_frames(self, block, frames, output, boxes=None):
        output["block"][block] = frames
        if self.include_simbox and boxes is not None:
            output["sim_box"][block] = boxes
