"""Pair potential and neighbour lists (gamdpy/interactions/).

``PairPotential`` keeps gamdpy's constructor and parameter conventions
(pair_potential.py:12-51): a potential function, ``params`` = [p0, p1, ...,
cut] as scalars or ntypes x ntypes arrays, ``max_num_nbs``.  Its kernels are
the CUDA ones of libgamdb200 (forces/virial/energy fused with the integrator);
``NbList2`` and ``NbListLinkedLists`` select the library's N^2 or cell-list
build, as ``compute_plan['nblist']`` does in gamdpy (pair_potential.py:89-94).
"""
import numpy as np

from . import _lib


class Interaction:
    """Abstract interaction (gamdpy/interactions/interaction.py:7-33)."""

    def check_datastructure_validity(self) -> bool:
        return True


class NbList2:
    """O(N^2) neighbour-list build (gamdpy/interactions/nblist.py:5-163).
    ``exclusions``: None or the (N, max_exclusions + 1) int32 table with the
    count last (Bonds.get_exclusions); excluded pairs never enter the list."""
    kind = _lib.NBLIST_NSQ

    def __init__(self, configuration, exclusions, max_num_nbs):
        self.N = configuration.N
        self.max_num_nbs = max_num_nbs
        self.exclusions = None
        if exclusions is not None:
            ex = np.ascontiguousarray(np.asarray(exclusions, dtype=np.int32))
            if ex.ndim != 2 or ex.shape[0] != self.N or ex.shape[1] < 2:
                raise ValueError(f"exclusions must be (N, max + 1) with the count last, got {ex.shape}")
            self.exclusions = ex


class NbListLinkedLists(NbList2):
    """Cell-list build (gamdpy/interactions/nblist_linked_lists.py:7-300)."""
    kind = _lib.NBLIST_CELLS


def _param_table(params_user):
    """(ntypes, ntypes, nparams) float32 table + max_cut, as
    PairPotential.convert_user_params (pair_potential.py:23-51)."""
    mats = []
    for p in params_user:
        if np.ndim(p) == 0:
            mats.append(np.ones((1, 1)) * float(p))
        else:
            mats.append(np.array(p, dtype=np.float32))
    nt = mats[0].shape[0]
    for m in mats:
        assert len(m.shape) == 2
        assert m.shape[0] == nt
        assert m.shape[1] == nt
    table = np.ascontiguousarray(np.stack([m.astype(np.float32) for m in mats], axis=-1))
    max_cut = np.float32(np.max(mats[-1]))
    return table, max_cut


class PairPotential(Interaction):
    """Pair potential over a neighbour list (gamdpy/interactions/pair_potential.py:9-268)."""

    def __init__(self, pairpotential_function, params, max_num_nbs, exclusions=None):
        self.pairpotential_function = pairpotential_function
        self.params_user = params
        self.exclusions = exclusions
        self.max_num_nbs = max_num_nbs
        self.nblist = None
        self._device = None

    def convert_user_params(self):
        table, max_cut = _param_table(self.params_user)
        nt = table.shape[0]
        rec = np.zeros((nt, nt), dtype="f," * table.shape[2])
        for i in range(nt):
            for j in range(nt):
                rec[i, j] = tuple(table[i, j])
        return rec, max_cut

    def table(self):
        return _param_table(self.params_user)

    def kernel_kind(self):
        """(potential kind, cutoff mode) of the CUDA kernel for this function."""
        f = self.pairpotential_function
        kind = getattr(f, "_gdb_kind", None)
        cutmode = getattr(f, "_gdb_cutmode", None)
        if kind is None or cutmode is None:
            raise NotImplementedError(
                "gamdpy_b200 evaluates pair potentials in CUDA; supported are LJ_12_6 and LJ_12_6_sigma_epsilon "
                "wrapped in apply_shifted_force_cutoff or apply_shifted_potential_cutoff "
                f"(got {getattr(f, '__name__', f)!r})")
        return kind, cutmode

    def evaluate_potential_function(self, r, types):
        table, _ = self.table()
        u, s, lap = self.pairpotential_function(r, table[types[0], types[1]])
        return u

    def make_nblist(self, configuration, compute_plan):
        if compute_plan["nblist"] == "N squared":
            self.nblist = NbList2(configuration, self.exclusions, self.max_num_nbs)
        elif compute_plan["nblist"] == "linked lists":
            self.nblist = NbListLinkedLists(configuration, self.exclusions, self.max_num_nbs)
        else:
            raise ValueError(f"No lblist called: {compute_plan['nblist']}. Use either 'N squared' or 'linked lists'")
        return self.nblist

    def configure_device(self, sim, configuration, compute_plan):
        """Send the potential and neighbour-list settings to a library handle."""
        kind, cutmode = self.kernel_kind()
        table, max_cut = self.table()
        nt_conf = int(np.max(configuration.ptype)) + 1 if configuration.N else 1
        if table.shape[0] < nt_conf:
            raise ValueError(f"parameter table has {table.shape[0]} types but the configuration uses {nt_conf}")
        sim.set_pair_potential(kind, cutmode, table)
        nbl = self.make_nblist(configuration, compute_plan)
        sim.set_nblist(nbl.kind, float(np.float32(compute_plan["skin"])), self.max_num_nbs)
        sim.set_exclusions(nbl.exclusions)
        self._device = sim
        self.max_cut = max_cut

    def check_datastructure_validity(self) -> bool:
        """Raise like pair_potential.py:78-82 when the list overflowed."""
        if self._device is None:
            return True
        nbflag = self._device.nbflag()
        if nbflag[1] != 0:
            raise RuntimeError(
                f"Neighbor-list is invalid. Try allocating space for more neighbors (max_num_nbs in PairPot "
                f"object). Allocated size: {self.max_num_nbs}, but {nbflag[1] + 1} neighbours found. {nbflag=}.")
        return True

    def get_nblist(self):
        """Neighbour list in gamdpy's layout (N, max_num_nbs+1), count last."""
        return self._device.nblist(self.max_num_nbs)


class Bonds(Interaction):
    """Fixed bonds between particles (gamdpy/interactions/bonds.py:12-150):
    ``bond_potential`` (harmonic_bond_function), ``potential_params`` one
    (r0, k) row per bond type, ``indices`` rows (i, j, bond type).  The bond
    forces are added per particle inside the library's fused step (each end
    evaluates its bonds: no atomics, the same sums in every run)."""

    def __init__(self, bond_potential, potential_params, indices):
        self.bond_potential = bond_potential
        self.potential_params = potential_params
        self.indices = indices
        self._device = None

    def _arrays(self):
        if getattr(self.bond_potential, "_gdb_bond", None) != "harmonic":
            raise NotImplementedError("gamdpy_b200 evaluates harmonic bonds (harmonic_bond_function) in CUDA; got "
                                      f"{getattr(self.bond_potential, '__name__', self.bond_potential)!r}")
        params = np.ascontiguousarray(np.array(self.potential_params, dtype=np.float32))
        if params.ndim != 2 or params.shape[1] < 2:
            raise ValueError("potential_params must hold one (r0, k) row per bond type")
        indices = np.ascontiguousarray(np.array(self.indices, dtype=np.int32))
        if indices.ndim != 2 or indices.shape[1] != 3:
            raise ValueError("indices must be rows (i, j, bond type)")
        if len(indices) and indices[:, -1].max() >= params.shape[0]:
            raise ValueError("a bond type has no parameter row")
        return indices, params[:, :2].copy()

    def get_exclusions(self, configuration, max_number_exclusions=20):
        """(N, max + 1) int32 table of every particle's bonded partners with
        the count last, the reference's format (bonds.py:137-150)."""
        exclusions = np.zeros((configuration.N, max_number_exclusions + 1), dtype=np.int32)
        for i, j, _ in self.indices:
            for a, b in ((i, j), (j, i)):
                if exclusions[a, -1] < max_number_exclusions:
                    exclusions[a, exclusions[a, -1]] = b
                exclusions[a, -1] += 1
        assert np.max(exclusions[:, -1]) <= max_number_exclusions
        return exclusions

    def configure_device(self, sim, configuration):
        indices, params = self._arrays()
        sim.set_bonds(indices, params)
        self._device = sim
