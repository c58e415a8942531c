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
    """O(N^2) neighbour-list build (gamdpy/interactions/nblist.py:5-163)."""
    kind = _lib.NBLIST_NSQ

    def __init__(self, configuration, exclusions, max_num_nbs):
        if exclusions is not None and len(exclusions) > 0:
            raise NotImplementedError("neighbour-list exclusions are outside the B200 hot path")
        self.N = configuration.N
        self.max_num_nbs = max_num_nbs


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
