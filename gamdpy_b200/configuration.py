"""Configuration, column arrays and lattices: gamdpy's data model.

Host-side mirror of gamdpy/configuration/Configuration.py, colarray.py,
make_lattice.py and unit_cells.py (same names, shapes, dtypes and column
order), so the particle state a user builds is laid out exactly as gamdpy's.
The device copy is owned by the simulation handle the configuration is
attached to; ``copy_to_device`` / ``copy_to_host`` move the state through the
library (``gdb_upload_state`` / ``gdb_download_state``).
"""
import numpy as np

from .simulation_boxes import Orthorhombic


def get_default_compute_flags():
    """gamdpy/simulation/get_default_compute_flags.py:2-5."""
    return {"U": True, "W": True, "K": True, "lapU": False, "Fsq": False, "stresses": False, "Vol": False,
            "Ptot": False}


class colarray:
    """Columns of (N, D) arrays stored in one (ncol, N, D) array
    (gamdpy/configuration/colarray.py:41-60)."""

    def __init__(self, column_names, size, dtype=np.float32, array=None):
        self.column_names = column_names
        self.dtype = dtype
        self.indices = {key: index for index, key in enumerate(column_names)}
        if isinstance(array, np.ndarray):
            self.array = array
        else:
            self.array = np.zeros((len(column_names), *size), dtype=dtype)
        self.shape = self.array.shape

    def __setitem__(self, key, data):
        self.array[self.indices[key]] = data

    def __getitem__(self, key):
        return self.array[self.indices[key]]

    def __repr__(self):
        return "colarray(" + str(tuple(self.indices.keys())) + ", " + repr(self.array.shape[1:]) + ")\n" + repr(
            self.array)

    def copy(self):
        return colarray(self.column_names, self.shape, self.dtype, self.array.copy())


class unit_cells:
    """gamdpy/configuration/unit_cells.py:1-15."""
    FCC = {"fractional_coordinates": [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]],
           "lattice_constants": [1.0, 1.0, 1.0]}
    BCC = {"fractional_coordinates": [[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]], "lattice_constants": [1.0, 1.0, 1.0]}
    SC = {"fractional_coordinates": [[0.0, 0.0, 0.0]], "lattice_constants": [1.0, 1.0, 1.0]}


def make_lattice(unit_cell, cells=None, rho=None):
    """Positions of a replicated unit cell centred in [-L/2, L/2) and the box
    vector (gamdpy/configuration/make_lattice.py:1-60: cells enumerated in C
    order, particles of a cell contiguous, float64)."""
    pos = np.asarray(unit_cell["fractional_coordinates"], dtype=np.float64)
    lat = np.asarray(unit_cell["lattice_constants"], dtype=np.float64)
    npc, D = pos.shape
    if cells is None:
        cells = [1] * D
    cells = [int(c) for c in cells]
    idx = np.stack(np.unravel_index(np.arange(int(np.prod(cells))), cells), axis=1).astype(np.float64)
    positions = (idx[:, None, :] + pos[None, :, :]).reshape(-1, D)
    positions *= lat
    box_vector = lat * np.array(cells, dtype=np.float64)
    if rho is not None:
        volume_per_particle = np.prod(box_vector) / len(positions)
        scale_factor = ((1.0 / rho) / volume_per_particle) ** (1.0 / 3.0)
        positions *= scale_factor
        box_vector *= scale_factor
    positions -= box_vector / 2.0
    return positions, box_vector


def generate_random_velocities(N, D, T, seed, m=1, dtype=np.float32):
    """Maxwell-Boltzmann velocities with the reference's exact RNG call order
    (gamdpy/configuration/Configuration.py:373-385): legacy np.random.seed,
    one np.random.normal per column, centre-of-mass drift removed per column."""
    v = np.zeros((N, D), dtype=dtype)
    np.random.seed(seed)
    for k in range(D):
        v[:, k] = np.random.normal(v[:, k], (T / m) ** 0.5)
        CM_drift = np.mean(m * v[:, k]) / np.mean(m)
        v[:, k] -= CM_drift
    return dtype(v)


class Configuration:
    """Particle vectors (r, v, f), scalars (U, W, [lapU], K, [Fsq], m), types,
    images and the simulation box (gamdpy/configuration/Configuration.py:16-146)."""

    scalar_parameters = ["m"]
    scalar_computables_interactions = ["U", "W", "lapU"]
    scalar_computables_integrator = ["K", "Fsq"]

    def __init__(self, D, N=None, type_names=None, compute_flags=None, ftype=np.float32, itype=np.int32):
        self.D = D
        self.N = N
        self.type_names = type_names
        self.compute_flags = get_default_compute_flags()
        if compute_flags is not None:
            for k in compute_flags:
                if k not in self.compute_flags:
                    raise ValueError("Unknown key in compute_flags:%s" % k)
                self.compute_flags[k] = compute_flags[k]
        self.vector_columns = ["r", "v", "f"]
        if self.compute_flags["stresses"]:
            raise NotImplementedError("compute_flags['stresses'] is outside the B200 hot path")
        self.num_cscalars = 0
        self.sid = {}
        self.scalar_columns = []
        for label in self.scalar_computables_interactions:
            if self.compute_flags[label]:
                self.sid[label] = len(self.scalar_columns)
                self.scalar_columns.append(label)
                self.num_cscalars += 1
        for label in self.scalar_computables_integrator:
            if self.compute_flags[label]:
                self.sid[label] = len(self.scalar_columns)
                self.scalar_columns.append(label)
        for label in self.scalar_parameters:
            self.sid[label] = len(self.scalar_columns)
            self.scalar_columns.append(label)
        self.simbox = None
        self.ftype = ftype
        self.itype = itype
        self._device = None  # gamdpy_b200._lib.Sim the state lives on, if any
        if self.N is not None:
            self._allocate_arrays()

    def _allocate_arrays(self):
        self.vectors = colarray(self.vector_columns, size=(self.N, self.D), dtype=self.ftype)
        self.scalars = np.zeros((self.N, len(self.scalar_columns)), dtype=self.ftype)
        self.r_im = np.zeros((self.N, self.D), dtype=self.itype)
        self.ptype = np.zeros(self.N, dtype=self.itype)

    def __repr__(self):
        return f"Configuration(D={self.D}, N={self.N}, compute_flags={self.compute_flags})"

    def __str__(self):
        if self.N is None:
            return f"{self.D} dimensional configuration. Particles not yet assigned."
        s = f"{self.N} particles in {self.D} dimensions. Number density (atomic): {self.N / self.get_volume():.3f}"
        return s

    def __setitem__(self, key, data):
        if self.N is None:
            if not isinstance(data, np.ndarray):
                raise TypeError("Number of particles, N, not determined yet, so assignment needs to be with a "
                                "numpy array")
            self.N = data.shape[0]
            self._allocate_arrays()
        if key in self.vector_columns:
            if isinstance(data, np.ndarray):
                N, D = data.shape
                if N != self.N:
                    raise ValueError(f"Inconsistent number of particles, {N} <> {self.N}")
                if D != self.D:
                    raise ValueError(f"Inconsistent number of dimensions, {D} <> {self.D}")
            self.vectors[key] = data
            return
        if key in self.scalar_columns:
            if isinstance(data, np.ndarray):
                (N,) = data.shape
                if N != self.N:
                    raise ValueError(f"Inconsistent number of particles, {N} <> {self.N}")
            self.scalars[:, self.sid[key]] = data
            return
        raise ValueError(f"Unknown key {key}. Vectors: {self.vector_columns}, Scalars: {self.scalar_columns}")

    def __getitem__(self, key):
        if key in self.vector_columns:
            return self.vectors[key]
        if key in self.scalar_columns:
            return self.scalars[:, self.sid[key]]
        raise ValueError(f"Unknown key {key}. Vectors: {self.vector_columns}, Scalars: {self.scalar_columns}")

    # --- host <-> device (Configuration.py:227-243) ----------------------
    def _attach(self, device):
        """Attach to a simulation handle.  The vectors, scalars and image
        arrays move into page-locked host memory (contents kept), so the
        copies to and from the device run at DMA speed; as in gamdpy, whose
        copy_to_host replaces these arrays (Configuration.py:236-243), views
        taken before this point no longer follow the configuration."""
        from . import _lib
        self._device = device
        for name, arr in (("vectors", self.vectors.array), ("scalars", self.scalars), ("r_im", self.r_im)):
            if getattr(self, "_pinned_" + name, None) is arr:
                continue
            pinned = _lib.pinned_empty(arr.shape, arr.dtype)
            if pinned is None:
                return
            pinned[...] = arr
            if name == "vectors":
                self.vectors.array = pinned
            else:
                setattr(self, name, pinned)
            setattr(self, "_pinned_" + name, pinned)

    def copy_to_device(self):
        """Upload the full state to the attached simulation handle."""
        if self._device is None:
            return
        self._device.set_box(self.simbox.lengths)
        self._device.upload(self["r"], self["v"], self["m"], self.ptype, self.r_im)

    def copy_to_host(self):
        """Download r, v, f, images and the per-particle scalars."""
        if self._device is None:
            return
        va, sc, im = self.vectors.array, self.scalars, self.r_im
        if (va.dtype == np.float32 and va.shape == (3, self.N, 3) and va.flags.c_contiguous and
                self.vector_columns == ["r", "v", "f"] and sc.dtype == np.float32 and sc.flags.c_contiguous and
                im.dtype == np.int32 and im.flags.c_contiguous and im.shape == (self.N, 3)):
            # one call straight into this configuration's arrays
            cols = [self.sid.get(k, -1) for k in ("U", "W", "lapU", "K", "Fsq", "m")]
            self._device.download_table(va, im, sc, cols)
            return
        vec = {k: self.vectors[k] for k in ("r", "v", "f")}
        im = self.r_im
        if all(a.dtype == np.float32 and a.flags.c_contiguous for a in vec.values()) and \
                im.dtype == np.int32 and im.flags.c_contiguous:
            self._device.download_into(vec["r"], vec["v"], vec["f"], im)
        else:
            st = self._device.download()
            for k in ("r", "v", "f"):
                self.vectors[k] = st[k]
            self.r_im[:] = st["r_im"]
        buf = getattr(self, "_scalar_buf", None)
        if buf is None or buf["U"].shape[0] != self.N:
            buf = {k: np.empty(self.N, np.float32) for k in ("U", "W", "lapU", "K", "Fsq")}
            self._scalar_buf = buf
        sc = self._device.download_scalars(buf)
        for k in ("U", "W", "lapU", "K", "Fsq"):
            if k in self.sid:
                self.scalars[:, self.sid[k]] = sc[k]

    # --- helpers -----------------------------------------------------------
    def get_potential_energy(self):
        return float(np.sum(self["U"]))

    def get_volume(self):
        return self.simbox.get_volume()

    def set_kinetic_temperature(self, temperature, ndofs=None):
        """Configuration.py:260-267."""
        if ndofs is None:
            ndofs = self.D * (self.N - 1)
        T_ = np.sum(np.dot(self["m"], np.sum(self["v"] ** 2, axis=1))) / ndofs
        if T_ == 0:
            raise ValueError("Cannot rescale velocities when all equal to zero")
        self["v"] *= (temperature / T_) ** 0.5

    def randomize_velocities(self, temperature, seed=None, ndofs=None):
        """Configuration.py:269-281."""
        if self.D is None:
            raise ValueError("Cannot randomize velocities. Start by assigning positions.")
        masses = self["m"]
        if np.any(masses == 0):
            raise ValueError("Cannot randomize velocities when any mass is zero")
        if temperature > 0.0:
            self["v"] = generate_random_velocities(self.N, self.D, T=temperature, seed=seed, m=self["m"])
            self.set_kinetic_temperature(temperature=temperature, ndofs=ndofs)
        else:
            self["v"] = np.zeros((self.N, self.D), np.float32)

    def make_lattice(self, unit_cell, cells, rho=None):
        """Configuration.py:283-306."""
        positions, box_vector = make_lattice(unit_cell=unit_cell, cells=cells, rho=rho)
        self["r"] = positions
        self.simbox = Orthorhombic(self.D, box_vector)

    def make_positions(self, N, rho):
        """Positions along the simple-cubic lines of ceil(N^(1/D)) particles,
        the reference's arithmetic (Configuration.py:308-361): coordinate d of
        particle i is (i mod p^(d+1)) / p^d with true division (p particles
        per line), so consecutive indices step one lattice spacing in x and a
        fraction of one in the other dimensions -- chains built from
        consecutive indices start with equal bond lengths -- then the centring
        offsets, the shift by int(p/2) and the scaling to density rho."""
        D = self.D
        ppl = float(np.ceil(pow(N, 1.0 / D)))
        box_length = pow(N / rho, 1.0 / D)
        idx = np.arange(N, dtype=np.float64)
        pos = np.empty((N, D), np.float64)
        pos[:, D - 1] = idx / ppl ** (D - 1)
        for d in range(D - 2, -1, -1):
            pos[:, d] = (idx % ppl ** (d + 1)) / ppl ** d
        remove = 0
        for d in range(1, D):
            remove += D ** (D - d)
            pos[:, d] -= remove / N
        pos -= np.array(D * [int(0.5 * ppl)])
        pos *= box_length / ppl
        self["r"] = pos
        self.simbox = Orthorhombic(D, np.array(D * [box_length]))

    def atomic_scale(self, density):
        actual_rho = self.N / self.get_volume()
        scale_factor = (actual_rho / density) ** (1 / 3)
        self.vectors["r"] *= scale_factor
        self.simbox.lengths *= scale_factor
