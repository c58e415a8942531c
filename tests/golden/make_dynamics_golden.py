"""Golden vectors of gamdpy's trajectory post-processing (tools/calc_dynamics.py).

Loads the reference's tools/calc_dynamics.py from its source tree (matplotlib,
which that module imports for its plotting helpers only, is not installed
here: an empty stand-in module takes its place) and runs calc_dynamics on a
seeded synthetic trajectory in the layout of the ConfigurationSaver output:
block frames (num_blocks, conf_per_block, 2, N, 3) float32 holding positions
inside the box and image counts, ptype, attrs dt and simbox_initial.

Run from the repository root:  python tests/golden/make_dynamics_golden.py
(the reference's source tree is read from /root/reference; GAMDPY_REF
overrides it).
"""
import importlib.util
import os
import sys
import types

import numpy as np

REF = os.path.join(os.environ.get("GAMDPY_REF", "/root/reference"), "gamdpy", "tools", "calc_dynamics.py")


class Trajectory(dict):
    def __init__(self, block, ptype, dt, box):
        super().__init__(block=block, ptype=ptype)
        self.attrs = {"dt": dt, "simbox_initial": box}


def synthetic(num_blocks=9, conf_per_block=6, n=96, seed=5):
    rng = np.random.default_rng(seed)
    box = np.array([6.0, 6.5, 7.0], np.float32)
    ptype = (rng.random(n) < 0.25).astype(np.int32)
    steps = num_blocks * conf_per_block
    walk = np.cumsum(rng.normal(0.0, 0.35, (steps, n, 3)), axis=0) + rng.uniform(-3, 3, (1, n, 3))
    img = np.floor(walk / box + 0.5)
    r = (walk - img * box).astype(np.float32)
    frames = np.zeros((num_blocks, conf_per_block, 2, n, 3), np.float32)
    frames[:, :, 0] = r.reshape(num_blocks, conf_per_block, n, 3)
    frames[:, :, 1] = img.reshape(num_blocks, conf_per_block, n, 3).astype(np.float32)
    return Trajectory(frames, ptype, 0.005, box)


def main():
    sys.modules.setdefault("matplotlib", types.ModuleType("matplotlib"))
    sys.modules.setdefault("matplotlib.pyplot", types.ModuleType("matplotlib.pyplot"))
    spec = importlib.util.spec_from_file_location("ref_calc_dynamics", REF)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    traj = synthetic()
    out = {"block": traj["block"], "ptype": traj["ptype"], "dt": traj.attrs["dt"],
           "simbox_initial": traj.attrs["simbox_initial"]}
    for tag, first, q in (("a", 1, 7.25), ("b", 0, np.array([6.0, 8.5]))):
        res = mod.calc_dynamics(traj, first, qvalues=q)
        out[f"{tag}_first_block"] = first
        out[f"{tag}_qvalues"] = np.asarray(res["qvalues"], np.float64)
        for k in ("times", "msd", "alpha2", "Fs", "count"):
            out[f"{tag}_{k}"] = res[k]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dynamics.npz")
    np.savez(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
