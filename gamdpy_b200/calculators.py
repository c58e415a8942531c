"""Radial distribution and structure factor calculators
(gamdpy/calculators/calculator_radial_distribution.py,
calculator_structure_factor.py).

Both compute on the B200 through libgamdb200.  When the configuration belongs
to a running Simulation the device-resident state is used directly (no host
copy); otherwise the host arrays are sent for the one call.
"""
import itertools
import math

import numpy as np

from . import _lib


class CalculatorRadialDistribution:
    """g(r) histograms per type pair over [0, r_max), r_max = min(L)/2 by
    default as in the reference (calculator_radial_distribution.py:12-185).
    ``r_max`` is an extension: a shorter range uses a cell search instead of
    all pairs.  Counts are exact integers, bit-identical to the reference's
    float64 histogram entries on the same positions."""

    def __init__(self, configuration, bins, compute_plan=None, ptype=None, r_max=None):
        if configuration.D != 3:
            raise NotImplementedError("gamdpy_b200 computes the RDF in D = 3")
        self.configuration = configuration
        self.ptype = np.asarray(ptype, np.int32) if ptype is not None else None
        self.bins = bins
        self.count = 0
        self.compute_plan = compute_plan
        self.r_max = r_max
        self.rdf_list = []
        pt = self.ptype if self.ptype is not None else configuration.ptype
        self.ntypes = int(np.max(pt)) + 1
        self.gr_bins = np.zeros((self.ntypes, self.ntypes, self.bins), dtype=np.float64)

    def _rmax(self):
        return 0.0 if self.r_max is None else float(self.r_max)

    def update(self):
        """Add the current configuration (calculator_radial_distribution.py:111-119)."""
        self.count += 1
        conf = self.configuration
        dev = conf._device
        if dev is not None and self.ptype is None and dev.ntypes == self.ntypes:
            out = np.zeros((self.ntypes, self.ntypes, self.bins), np.uint64)
            dev.rdf_update(self.bins, self._rmax(), out)
        else:
            pt = self.ptype if self.ptype is not None else conf.ptype
            out = _lib.rdf_compute(conf["r"], pt, conf.simbox.lengths, self.ntypes, self.bins, self._rmax())
        self.rdf_list.append(out.astype(np.float64))

    def read(self):
        """Normalised g(r) (calculator_radial_distribution.py:121-159)."""
        bins = self.rdf_list[0].shape[2]
        min_box_dim = np.min(self.configuration.simbox.lengths)
        r_max = (min_box_dim / 2) if self.r_max is None else self.r_max
        bin_width = r_max / bins
        rdf_ptype = np.array(self.rdf_list)
        rho = self.configuration.N / np.prod(self.configuration.simbox.lengths)
        D = self.configuration.D
        n = (D - 1) // 2
        unit_hypersphere_volume = (2 ** D * math.pi ** n * math.factorial(n)) / math.factorial(D)
        for i in range(bins):
            r_outer = (i + 1) * bin_width
            r_inner = i * bin_width
            shell_volume = unit_hypersphere_volume * (r_outer ** D - r_inner ** D)
            expected_num = rho * shell_volume
            rdf_ptype[:, :, :, i] /= (expected_num * self.configuration.N)
        rdf = rdf_ptype.sum(axis=1).sum(axis=1)
        ptype = self.ptype if self.ptype is not None else self.configuration.ptype
        for j in range(rdf_ptype.shape[1]):
            n_j = np.sum(ptype == j) / len(ptype)
            rdf_ptype[:, j, :, :] /= n_j
        for k in range(rdf_ptype.shape[2]):
            n_k = np.sum(ptype == k) / len(ptype)
            rdf_ptype[:, :, k, :] /= n_k
        distances = np.arange(0, bins) * bin_width
        return {"distances": distances, "rdf": rdf, "rdf_ptype": rdf_ptype, "ptype": ptype}

    def save_average(self, output_filename="rdf.dat", save_ptype=False):
        rdf_dict = self.read()
        rdf_total = np.mean(rdf_dict["rdf"], axis=0)
        rdf_ij, header_ij = [], " "
        for i in range(rdf_dict["rdf_ptype"].shape[1]):
            for j in range(rdf_dict["rdf_ptype"].shape[2]):
                rdf_ij.append(np.mean(rdf_dict["rdf_ptype"][:, i, j, :], axis=0))
                header_ij += f"g[{i}-{j}](r) "
        np.savetxt(output_filename, np.array([rdf_dict["distances"], rdf_total, *rdf_ij]).T,
                   header=f"r g(r) {header_ij} ptype")


class CalculatorStructureFactor:
    """rho_q = N_f^-1/2 sum_n f_n exp(i q.r_n), S(q) = |rho_q|^2 for
    q = 2 pi n / L (calculator_structure_factor.py:9-276).  Every backend name
    of the reference is accepted; all of them compute on the B200 with float64
    accumulation."""

    BACKENDS = ["CPU multi core", "CPU single core", "GPU"]

    def __init__(self, configuration, n_vectors=None, atomic_form_factors=None, backend="GPU"):
        if backend not in self.BACKENDS:
            raise ValueError(f"Unknown backend, {backend}. The known backends are {self.BACKENDS}.")
        if configuration.D != 3:
            raise NotImplementedError("gamdpy_b200 computes S(q) in D = 3")
        self.update_count = 0
        self.configuration = configuration
        self.L = configuration.simbox.lengths.copy()
        if n_vectors is not None:
            self.n_vectors = np.array(n_vectors)
            if self.n_vectors.shape[1] != configuration.D:
                raise ValueError("n_vectors must have the same number of columns as the number of dimensions.")
            self.q_vectors = np.array(2 * np.pi * self.n_vectors / self.L, dtype=np.float32)
            self.q_lengths = np.linalg.norm(self.q_vectors, axis=1)
            self.sum_S_q = np.zeros_like(self.q_lengths)
        self.atomic_form_factors = atomic_form_factors
        if atomic_form_factors is None:
            self.atomic_form_factors = np.ones(configuration.N, dtype=np.float32)
        self._unit_ff = atomic_form_factors is None
        self.list_of_rho_q = []
        self.list_of_rho_S_q = []

    def generate_q_vectors(self, q_max):
        """n in [0, n_max)^D without the zero vector, |q| < q_max
        (calculator_structure_factor.py:114-129)."""
        D = self.configuration.D
        if q_max < 0.0:
            raise ValueError(f"{q_max=} must be positive")
        n_max = int(np.ceil(q_max * max(self.L) / (2 * np.pi)))
        n_vectors = np.array(list(itertools.product(range(n_max), repeat=D)), dtype=int)[1:]
        self.q_vectors = np.array(2 * np.pi * n_vectors / self.L, dtype=np.float32)
        selection = np.linalg.norm(self.q_vectors, axis=1) < q_max
        self.q_vectors = self.q_vectors[selection]
        self.n_vectors = n_vectors[selection]
        self.q_lengths = np.linalg.norm(self.q_vectors, axis=1)
        self.sum_S_q = np.zeros_like(self.q_lengths)

    def update(self):
        """Add the current configuration (calculator_structure_factor.py:205-213)."""
        conf = self.configuration
        if not np.allclose(self.L, conf.simbox.lengths):
            raise ValueError("Box length has changed. Recreate the S(q) object.")
        ff = None if self._unit_ff else np.asarray(self.atomic_form_factors, np.float32)
        if conf._device is not None:
            rho_q = conf._device.sq_update(self.n_vectors, ff)
        else:
            rho_q = _lib.sq_compute(conf["r"], self.L, self.n_vectors, ff)
        self.list_of_rho_q.append(rho_q)
        s = np.abs(rho_q) ** 2
        self.list_of_rho_S_q.append(s)
        self.sum_S_q = self.sum_S_q + s
        self.update_count += 1

    def read(self, bins):
        """Binned or raw S(q) (calculator_structure_factor.py:216-268)."""
        if isinstance(bins, int):
            q_bins = np.linspace(0, np.max(self.q_lengths), bins + 1)
            q_binned = np.zeros(bins, dtype=np.float32)
            S_q_binned = np.zeros(bins, dtype=np.float32)
            q_in_bin = np.zeros(bins, dtype=int)
            for i in range(bins):
                mask = (q_bins[i] <= self.q_lengths) & (self.q_lengths < q_bins[i + 1])
                if np.sum(mask) == 0:
                    continue
                q_binned[i] = np.mean(self.q_lengths[mask])
                S_q_binned[i] = np.mean(self.sum_S_q[mask] / self.update_count)
                q_in_bin[i] = np.sum(mask)
            mask = q_in_bin > 0
            return {"|q|": q_binned[mask], "S(|q|)": S_q_binned[mask], "q_vectors_in_bin": q_in_bin[mask]}
        elif bins is None:
            return {"q": self.q_vectors, "|q|": self.q_lengths, "S(q)": self.sum_S_q / self.update_count,
                    "rho_q": np.array(self.list_of_rho_q), "n_vectors": self.n_vectors,
                    "atomic_form_factors": self.atomic_form_factors}
        raise ValueError("bins must be an integer.")

    def save_average(self, bins=None, output_filename="sq.dat"):
        if bins is None:
            bins = 100
        d = self.read(bins)
        np.savetxt(output_filename, np.c_[d["|q|"], d["S(|q|)"]], header="|q| S(|q|)")
