"""Helpers from gamdpy/misc: temperature schedules and scalar extraction."""
import numpy as np

from . import _lib


def make_function_constant(value):
    """Function returning a constant (misc/make_function.py:6-13)."""
    value = np.float32(value)

    def function(x):
        return value

    function._gdb_tfunc = _lib.TFUNC_CONSTANT
    function._gdb_tparams = [float(value)]
    return function


def make_function_ramp(value0, x0, value1, x1):
    """value0 for x < x0, linear to value1 at x1, value1 after
    (misc/make_function.py:16-34)."""
    value0, x0, value1, x1 = np.float32(value0), np.float32(x0), np.float32(value1), np.float32(x1)
    alpha = (value1 - value0) / (x1 - x0)

    def function(x):
        if x < x0:
            return value0
        if x < x1:
            return value0 + (x - x0) * alpha
        return value1

    function._gdb_tfunc = _lib.TFUNC_RAMP
    function._gdb_tparams = [float(value0), float(x0), float(value1), float(x1)]
    return function


def extract_scalars(data, column_list, first_block=0, D=3):
    """Columns of the ScalarSaver output, flattened over blocks and saves
    (misc/extract_scalars.py:1-51)."""
    try:
        scalar_names = data.attrs["scalar_names"]
    except KeyError:
        scalar_names = data.attrs["scalars_names"]
    column_indices = {name: index for index, name in enumerate(scalar_names)}
    return tuple(data["scalars"][first_block:, :, column_indices[c]].flatten() for c in column_list)
