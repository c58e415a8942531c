"""Generate golden fixtures by running the reference gamdpy on the CPU.

This script is test infrastructure.  It needs a checkout of gamdpy (default
``/root/reference``, override with ``GAMDPY_REF``) and is only run in a
container that has one; the GPU box never runs it.  Its outputs are the
``*.npz`` files beside it, which the tests read.

How gamdpy runs here: the numba CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``,
``NUMBA_DISABLE_JIT=1``, as gamdpy's own ``examples/minimal_cpu.py:9-11``
does), with ``gridsync=False`` and small ``pb`` so that every kernel of the
reference runs in its kernel-launch form (``Simulation.py:330-346``).  h5py and
matplotlib are absent from the image, so tiny in-memory stand-ins are put in
``sys.modules`` before gamdpy is imported (gamdpy imports them at
``simulation/Simulation.py:20`` and ``interactions/pair_potential.py:5``).

Two cases need compiled-numba typing rather than the simulator's numpy typing
(the RDF bin index, ``calculator_radial_distribution.py:81-105``, promotes to
float64 under numba).  Those are generated by ``rdf_numba_typed`` below, which
compiles the reference's own ``dist_sq_function`` with ``numba.njit`` and
evaluates the kernel's binning expressions under numba's typing rules.

S(q) uses gamdpy's own CPU backend (``calculator_structure_factor.py:185-196``)
in a separate process without the simulator.

Usage:  python tests/golden/make_golden.py [case ...]
"""
import math
import os
import sys
import time
import subprocess
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("GAMDPY_REF", "/root/reference")


# --------------------------------------------------------------------------
# stand-ins for the two packages gamdpy imports but the image lacks
# --------------------------------------------------------------------------
def _install_stubs():
    h5 = types.ModuleType("h5py")

    class File(dict):
        def __init__(self, *a, **k):
            super().__init__()
            self.attrs = {}

        def create_dataset(self, name, data=None, shape=None, dtype=None, chunks=None, **k):
            if data is None:
                data = np.zeros(shape, dtype=dtype)
            self[name] = np.array(data, dtype=dtype) if dtype is not None else np.array(data)
            return self[name]

        def create_group(self, name):
            g = File()
            self[name] = g
            return g

        def close(self):
            pass

    h5.File = File
    sys.modules["h5py"] = h5
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt


def _import_gamdpy(simulator=True):
    if simulator:
        os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
        os.environ["NUMBA_DISABLE_JIT"] = "1"
    _install_stubs()
    sys.path.insert(0, REF)
    import warnings
    warnings.filterwarnings("ignore")
    import gamdpy as gp
    return gp


# --------------------------------------------------------------------------
# inputs (seeded; stored in every fixture so tests never regenerate them)
# --------------------------------------------------------------------------
def lj_fcc_input(cells, rho, seed, jitter):
    """FCC lattice (gamdpy's make_lattice layout) + uniform jitter, permuted."""
    from_ref = _import_gamdpy_cached()
    pos, box = from_ref.configuration.make_lattice(from_ref.unit_cells.FCC, cells=cells, rho=rho)
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-jitter, jitter, pos.shape)
    pos = pos[rng.permutation(len(pos))]
    # wrap into [-L/2, L/2)
    pos = pos - box * np.round(pos / box)
    return pos.astype(np.float32), np.asarray(box, np.float32)


_GP = None


def _import_gamdpy_cached():
    global _GP
    if _GP is None:
        _GP = _import_gamdpy(simulator=True)
    return _GP


KA_SIG = np.array([[1.0, 0.8], [0.8, 0.88]], np.float32)
KA_EPS = np.array([[1.0, 1.5], [1.5, 0.5]], np.float32)
KA_CUT = (2.5 * KA_SIG).astype(np.float32)


def ka_types(n, seed):
    rng = np.random.default_rng(seed + 1)
    t = np.zeros(n, np.int32)
    t[rng.permutation(n)[: n // 5]] = 1
    return t


def make_conf(gp, pos, box, ptype=None, lapU=True, fsq=True):
    conf = gp.Configuration(D=3, compute_flags={"lapU": lapU, "Fsq": fsq})
    conf["r"] = pos.copy()
    conf.simbox = gp.Orthorhombic(3, box)
    conf["m"] = 1.0
    if ptype is not None:
        conf.ptype[:] = ptype
    return conf


def plan(nblist, skin, pb=4):
    return {"pb": pb, "tp": 1, "skin": np.float32(skin), "UtilizeNIII": False,
            "gridsync": False, "nblist": nblist}


def sorted_csr(nbl):
    """(N, max+1) gamdpy list -> CSR of per-row sorted neighbour ids."""
    counts = nbl[:, -1].astype(np.int32)
    rows = [np.sort(nbl[i, : counts[i]]) for i in range(len(nbl))]
    return counts, np.concatenate(rows).astype(np.int32)


# --------------------------------------------------------------------------
# case: force/energy evaluation over a neighbour list (Evaluator semantics)
# --------------------------------------------------------------------------
def eval_case(name, pos, box, ptype, params, cutoff, nblist_kind, skin, max_nbs):
    gp = _import_gamdpy_cached()
    conf = make_conf(gp, pos, box, ptype)
    fn = {"SF": gp.apply_shifted_force_cutoff, "SP": gp.apply_shifted_potential_cutoff}[cutoff]
    pp = gp.PairPotential(fn(gp.LJ_12_6_sigma_epsilon), params=params, max_num_nbs=max_nbs)
    cp = plan(nblist_kind, skin)
    flags = gp.get_default_compute_flags()
    flags.update({"lapU": True, "Fsq": True})
    kernel, iparams = gp.add_interactions_list(conf, [pp], compute_plan=cp, compute_flags=flags)
    conf.copy_to_device()
    t0 = time.time()
    kernel(0, conf.d_vectors, conf.d_scalars, conf.d_ptype, conf.simbox.d_data, iparams)
    conf.copy_to_host()
    nbl = pp.nblist.d_nblist.copy_to_host()
    nbflag = pp.nblist.d_nbflag.copy_to_host()
    counts, flat = sorted_csr(nbl)
    print(f"{name}: {time.time() - t0:.1f}s  N={len(pos)} mean nbs={counts.mean():.2f} nbflag={nbflag}")
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        r=pos, box=box, ptype=conf.ptype, sigma=np.asarray(params[0], np.float32),
        epsilon=np.asarray(params[1], np.float32), cut=np.asarray(params[2], np.float32),
        cutoff=cutoff, nblist=nblist_kind, skin=np.float32(skin),
        nb_counts=counts, nb_flat=flat, f=conf["f"], U=conf["U"], W=conf["W"],
        lapU=conf["lapU"], nbflag=nbflag,
    )


def case_lj256_sf():
    pos, box = lj_fcc_input([4, 4, 4], 0.973, seed=0, jitter=0.1)
    eval_case("lj256_sf", pos, box, None, [1.0, 1.0, 2.5], "SF", "N squared", 0.5, 300)


def case_lj256_sp():
    pos, box = lj_fcc_input([4, 4, 4], 0.973, seed=0, jitter=0.1)
    eval_case("lj256_sp", pos, box, None, [1.0, 1.0, 2.5], "SP", "N squared", 0.5, 300)


def case_ka1372_cells():
    pos, box = lj_fcc_input([7, 7, 7], 1.2, seed=3, jitter=0.05)
    t = ka_types(len(pos), 3)
    eval_case("ka1372_cells", pos, box, t, [KA_SIG, KA_EPS, KA_CUT], "SF", "linked lists", 0.3, 300)


# --------------------------------------------------------------------------
# case: short trajectories through Simulation (NVE / NVT + runtime actions)
# --------------------------------------------------------------------------
def traj_case(name, pos, box, ptype, vel, params, integrator, nblist_kind, skin, blocks, steps,
              every, reset):
    gp = _import_gamdpy_cached()
    conf = make_conf(gp, pos, box, ptype, lapU=False, fsq=False)
    conf["v"] = vel
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon),
                          params=params, max_num_nbs=300)
    if integrator[0] == "NVE":
        integ = gp.integrators.NVE(dt=integrator[1])
    else:
        integ = gp.integrators.NVT(temperature=integrator[2], tau=integrator[3], dt=integrator[1])
    actions = [gp.ScalarSaver(every)]
    if reset:
        actions.append(gp.MomentumReset(reset))
    r0, v0 = conf["r"].copy(), conf["v"].copy()
    t0 = time.time()
    sim = gp.Simulation(conf, pp, integ, actions, num_timeblocks=blocks, steps_per_timeblock=steps,
                        compute_plan=plan(nblist_kind, skin), storage="memory", timing=False)
    xi_after_test = integ.d_thermostat_state.copy_to_host() if integrator[0] == "NVT" else np.zeros(2)
    for _ in sim.run_timeblocks():
        pass
    nbflag = pp.nblist.d_nbflag.copy_to_host()
    xi = integ.d_thermostat_state.copy_to_host() if integrator[0] == "NVT" else np.zeros(2)
    print(f"{name}: {time.time() - t0:.1f}s  nbflag={nbflag} xi={xi}")
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        r0=r0, v0=v0, box=box, ptype=conf.ptype,
        sigma=np.asarray(params[0], np.float32), epsilon=np.asarray(params[1], np.float32),
        cut=np.asarray(params[2], np.float32), integrator=integrator[0],
        dt=np.float32(integrator[1]),
        temperature=np.float32(integrator[2] if integrator[0] == "NVT" else 0),
        tau=np.float32(integrator[3] if integrator[0] == "NVT" else 0),
        nblist=nblist_kind, skin=np.float32(skin), blocks=blocks, steps=steps,
        every=every, reset=reset, r=conf["r"], v=conf["v"], f=conf["f"], r_im=conf.r_im,
        U=conf["U"], W=conf["W"], K=conf["K"], scalars=sim.output["scalars"],
        scalar_names=np.array(sim.output.attrs["scalar_names"]), xi_after_test=xi_after_test,
        thermostat_state=xi, nbflag=nbflag,
    )


def mb_velocities(n, T, seed):
    """gamdpy's generate_random_velocities + set_kinetic_temperature
    (Configuration.py:373-385, 260-267), called through gamdpy itself."""
    gp = _import_gamdpy_cached()
    c = gp.Configuration(D=3)
    c["r"] = np.zeros((n, 3), np.float32)
    c["m"] = 1.0
    c.randomize_velocities(temperature=T, seed=seed)
    return c["v"].copy()


def case_lj256_nve():
    pos, box = lj_fcc_input([4, 4, 4], 0.973, seed=0, jitter=0.1)
    vel = mb_velocities(len(pos), 0.7, seed=0)
    traj_case("lj256_nve", pos, box, None, vel, [1.0, 1.0, 2.5], ("NVE", 0.005), "N squared", 0.5,
              blocks=2, steps=8, every=2, reset=4)


def case_ka1372_nvt():
    pos, box = lj_fcc_input([7, 7, 7], 1.2, seed=3, jitter=0.05)
    t = ka_types(len(pos), 3)
    vel = mb_velocities(len(pos), 0.45, seed=3)
    traj_case("ka1372_nvt", pos, box, t, vel, [KA_SIG, KA_EPS, KA_CUT], ("NVT", 0.005, 0.45, 0.2),
              "linked lists", 0.3, blocks=1, steps=6, every=2, reset=0)


# --------------------------------------------------------------------------
# case: RDF.  Simulator run of the kernel + numba-typed evaluation.
# --------------------------------------------------------------------------
def rdf_numba_typed(r, box, ptype, bins):
    """Compiled-numba evaluation of the RDF kernel's arithmetic
    (calculator_radial_distribution.py:81-105) with the reference's own
    dist_sq_function (simulation_boxes/orthorhombic.py:59-73)."""
    import numba
    sys.path.insert(0, REF)
    _install_stubs()
    import importlib
    ortho = importlib.import_module("gamdpy.simulation_boxes.orthorhombic")
    dist_sq_function = numba.njit(ortho.Orthorhombic(3, box).get_dist_sq_function())

    @numba.njit
    def kernel(r, sim_box, ptype, gr):
        num_part = r.shape[0]
        bins = gr.shape[2]
        min_box_dim = min(sim_box[0], min(sim_box[1], sim_box[2]))
        bin_width = (min_box_dim / 2) / bins
        for i in range(num_part):
            for j in range(num_part):
                if j != i:
                    dist_sq = dist_sq_function(r[j], r[i], sim_box)
                    if dist_sq < (min_box_dim / 2) ** 2:
                        dist = math.sqrt(dist_sq)
                        if dist < min_box_dim / 2:
                            bin_index = int(dist / bin_width)
                            gr[ptype[i], ptype[j], bin_index] += 1

    nt = int(ptype.max()) + 1
    gr = np.zeros((nt, nt, bins), np.float64)
    kernel(r.astype(np.float32), box.astype(np.float32), ptype.astype(np.int32), gr)
    return gr


def case_rdf():
    out = {}
    typed = np.load(os.path.join(HERE, "rdf_typed.npz"))
    for tag, src in (("lj256", "lj256_sf"), ("ka1372", "ka1372_cells")):
        d = np.load(os.path.join(HERE, f"{src}.npz"))
        out[f"{tag}_r"] = d["r"]
        out[f"{tag}_box"] = d["box"]
        out[f"{tag}_ptype"] = d["ptype"]
        out[f"{tag}_bins_numba"] = typed[f"{tag}_bins_numba"]
    # simulator run of the reference kernel on the small case
    gp = _import_gamdpy_cached()
    d = np.load(os.path.join(HERE, "lj256_sf.npz"))
    conf = make_conf(gp, d["r"], d["box"])
    conf.copy_to_device()
    calc = gp.CalculatorRadialDistribution(conf, bins=100, compute_plan=plan("N squared", 0.5))
    t0 = time.time()
    calc.update()
    out["lj256_bins_simulator"] = calc.rdf_list[0]
    out["lj256_read_rdf"] = calc.read()["rdf"]
    print(f"rdf: simulator {time.time() - t0:.1f}s; numba-typed vs simulator max diff "
          f"{np.abs(out['lj256_bins_simulator'] - out['lj256_bins_numba']).max()}")
    np.savez_compressed(os.path.join(HERE, "rdf.npz"), bins=100, **out)


def case_sq():
    """Runs in a fresh process without the simulator: gamdpy's CPU backend."""
    code = f"""
import sys, numpy as np
sys.path.insert(0, {HERE!r})
import make_golden as mg
gp = mg._import_gamdpy(simulator=False)
d = np.load({os.path.join(HERE, 'ka1372_cells.npz')!r})
conf = gp.Configuration(D=3)
conf['r'] = d['r'].copy()
conf.simbox = gp.Orthorhombic(3, d['box'])
conf['m'] = 1.0
res = {{}}
for backend in ('CPU multi core', 'CPU single core'):
    calc = gp.CalculatorStructureFactor(conf, backend=backend)
    calc.generate_q_vectors(q_max=9.0)
    calc.update()
    raw = calc.read(None)
    key = backend.split()[1]
    res[key + '_rho_q'] = raw['rho_q'][0]
    res[key + '_S'] = raw['S(q)']
    res['q'] = raw['q']; res['n_vectors'] = raw['n_vectors']
    binned = calc.read(20)
    res[key + '_Sbin'] = binned['S(|q|)']; res[key + '_qbin'] = binned['|q|']
ff = np.where(d['ptype'] == 1, 0.5, 1.0).astype(np.float32)
calc = gp.CalculatorStructureFactor(conf, atomic_form_factors=ff, backend='CPU multi core')
calc.generate_q_vectors(q_max=6.0)
calc.update()
raw = calc.read(None)
res['ff'] = ff; res['ff_q'] = raw['q']; res['ff_rho_q'] = raw['rho_q'][0]
np.savez_compressed({os.path.join(HERE, 'sq.npz')!r}, r=d['r'], box=d['box'], ptype=d['ptype'], **res)
print('sq: q vectors', len(res['q']))
"""
    subprocess.run([sys.executable, "-c", code], check=True)


def case_known_answers():
    """Known-answer values of the reference's own tests, recomputed by calling
    gamdpy (tests/test_potential_functions.py:9-10, tests/test_simbox.py:5-50)
    plus the two cutoff wrappers at a grid of distances."""
    gp = _import_gamdpy(simulator=False)
    res = {}
    res["lj_12_6_1_23"] = np.array(gp.LJ_12_6(1, [2, 3]), np.float64)
    res["lj_se_1_23"] = np.array(gp.LJ_12_6_sigma_epsilon(1, [2, 3]), np.float64)
    rr = np.linspace(0.8, 2.6, 37).astype(np.float32)
    prm = np.array([1.0, 1.0, 2.5], np.float32)
    prm_ka = np.array([0.8, 1.5, 2.0], np.float32)
    for tag, fn in (("sf", gp.apply_shifted_force_cutoff), ("sp", gp.apply_shifted_potential_cutoff)):
        pot = fn(gp.LJ_12_6_sigma_epsilon)
        res[f"{tag}_r"] = rr
        res[f"{tag}_lj"] = np.array([pot(np.float32(x), prm) for x in rr], np.float64)
        res[f"{tag}_ka"] = np.array([pot(np.float32(x), prm_ka) for x in rr], np.float64)
    box = gp.Orthorhombic(D=3, lengths=np.array([3, 4, 5]))
    dr = np.zeros(3)
    res["mic_dist_sq"] = box.get_dist_sq_dr_function()(np.array([2.5, 3, 4]), np.array([0.5, 0.5, 0.5]),
                                                          box.lengths, dr)
    res["mic_dr"] = dr
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), **res)
    print("known answers:", {k: v for k, v in res.items() if v.size < 5})


# --------------------------------------------------------------------------
# case: molecules -- harmonic bonds (interactions/bonds.py) with the bonded
# pairs excluded from the pair potential's neighbour list, as the reference's
# examples/LJchain.py sets them up: chains of 10 beads on gamdpy's simple
# cubic positions, two bond types (r0, k) alternating along the chains
# --------------------------------------------------------------------------
CHAIN_BONDS = [[1.0, 3000.0], [1.1, 2000.0]]


class _KernelCuda:
    """The running simulated kernel's cuda module.  The reference's bond
    calculator (interactions/bonds.py:102-135) is compiled with numba.njit,
    so under the simulator its ``cuda`` global is the module-level API, which
    has no per-thread local arrays; this proxy hands it the kernel's own."""

    def __getattr__(self, name):
        from numba import cuda
        from numba.cuda.simulator.kernel import _get_kernel_context
        ctx = _get_kernel_context()
        return getattr(ctx if ctx is not None else cuda, name)


def chain_system(gp, n, rho, seed):
    import gamdpy.interactions.bonds as bonds_module
    bonds_module.cuda = _KernelCuda()
    conf = gp.Configuration(D=3, compute_flags={"lapU": True, "Fsq": True})
    conf.make_positions(N=n, rho=rho)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=1.0, seed=seed)
    indices = [[i, i + 1, i % 2] for i in range(n - 1) if i % 10 != 9]
    bonds = gp.Bonds(gp.harmonic_bond_function, CHAIN_BONDS, indices)
    excl = bonds.get_exclusions(conf)
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          exclusions=excl, max_num_nbs=300)
    return conf, bonds, excl, pp, np.array(indices, np.int32)


def chain_eval_case(name, n, nblist_kind):
    gp = _import_gamdpy_cached()
    conf, bonds, excl, pp, indices = chain_system(gp, n, 1.0, seed=4)
    cp = plan(nblist_kind, 0.5)
    flags = gp.get_default_compute_flags()
    flags.update({"lapU": True, "Fsq": True})
    kernel, iparams = gp.add_interactions_list(conf, [pp, bonds], compute_plan=cp, compute_flags=flags)
    conf.copy_to_device()
    t0 = time.time()
    kernel(0, conf.d_vectors, conf.d_scalars, conf.d_ptype, conf.simbox.d_data, iparams)
    conf.copy_to_host()
    nbl = pp.nblist.d_nblist.copy_to_host()
    counts, flat = sorted_csr(nbl)
    print(f"{name}: {time.time() - t0:.1f}s  N={n} mean nbs={counts.mean():.2f}")
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), r=conf["r"], box=conf.simbox.lengths, v=conf["v"],
                        bond_indices=indices, bond_params=np.array(CHAIN_BONDS, np.float32), exclusions=excl,
                        nblist=nblist_kind, skin=np.float32(0.5), nb_counts=counts, nb_flat=flat, f=conf["f"],
                        U=conf["U"], W=conf["W"], lapU=conf["lapU"])


def case_chain200_bonds():
    chain_eval_case("chain200_bonds", 200, "N squared")


def case_chain1200_cells():
    chain_eval_case("chain1200_cells", 1200, "linked lists")


def case_chain200_nve():
    """8 NVE steps (dt 0.002) of the chain system through Simulation with
    [PairPotential, Bonds], ScalarSaver every 2 steps."""
    gp = _import_gamdpy_cached()
    conf, bonds, excl, pp, indices = chain_system(gp, 200, 1.0, seed=4)
    r0, v0 = conf["r"].copy(), conf["v"].copy()
    t0 = time.time()
    sim = gp.Simulation(conf, [pp, bonds], gp.integrators.NVE(dt=0.002), [gp.ScalarSaver(2)], num_timeblocks=1,
                        steps_per_timeblock=8, compute_plan=plan("N squared", 0.5), storage="memory", timing=False)
    for _ in sim.run_timeblocks():
        pass
    print(f"chain200_nve: {time.time() - t0:.1f}s")
    np.savez_compressed(os.path.join(HERE, "chain200_nve.npz"), r0=r0, v0=v0, box=conf.simbox.lengths,
                        bond_indices=indices, bond_params=np.array(CHAIN_BONDS, np.float32), exclusions=excl,
                        dt=np.float32(0.002), steps=8, every=2, r=conf["r"], v=conf["v"], f=conf["f"],
                        r_im=conf.r_im, U=conf["U"], W=conf["W"], scalars=sim.output["scalars"],
                        scalar_names=np.array(sim.output.attrs["scalar_names"]))


# cases that must see compiled numba (no simulator) run with simulator=False
NO_SIMULATOR = {"known_answers", "rdf_typed"}


def case_rdf_typed():
    out = {}
    for tag, src in (("lj256", "lj256_sf"), ("ka1372", "ka1372_cells")):
        d = np.load(os.path.join(HERE, f"{src}.npz"))
        out[f"{tag}_bins_numba"] = rdf_numba_typed(d["r"], d["box"], d["ptype"], 100)
    np.savez_compressed(os.path.join(HERE, "rdf_typed.npz"), **out)
    print("rdf_typed: done")


def case_lj256_npt():
    """NPT_Atomic (integrators/NPT_Atomic.py) on an LJ liquid started from a
    jittered FCC lattice well above the target pressure, so the barostat
    moves the box from the first step: two timeblocks of 8 steps with
    ScalarSaver(2) saving U, W, K and Vol and ConfigurationSaver frames with
    their boxes (include_simbox).  The thermostat and barostat
    states are read from gamdpy's device arrays after the kernel test step
    and after the run."""
    gp = _import_gamdpy_cached()
    pos, box = lj_fcc_input([4, 4, 4], 0.973, seed=5, jitter=0.1)
    vel = mb_velocities(len(pos), 2.0, seed=5)
    conf = gp.Configuration(D=3, compute_flags={"Vol": True})
    conf["r"] = pos.copy()
    conf.simbox = gp.Orthorhombic(3, box)
    conf["m"] = 1.0
    conf["v"] = vel
    params = [1.0, 1.0, 2.5]
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=params, max_num_nbs=300)
    T, tau, P, tau_p, dt = 2.0, 0.4, 4.7, 2.0, 0.004
    integ = gp.integrators.NPT_Atomic(temperature=T, tau=tau, pressure=P, tau_p=tau_p, dt=dt)
    r0, v0 = conf["r"].copy(), conf["v"].copy()
    t0 = time.time()
    sim = gp.Simulation(conf, pp, integ, [gp.ConfigurationSaver(include_simbox=True), gp.ScalarSaver(2)],
                        num_timeblocks=2, steps_per_timeblock=8, compute_plan=plan("N squared", 0.5),
                        storage="memory", timing=False)
    ts_test = integ.d_thermostat_state.copy_to_host()
    bs_test = integ.d_barostat_state.copy_to_host()
    for _ in sim.run_timeblocks():
        pass
    ts = integ.d_thermostat_state.copy_to_host()
    bs = integ.d_barostat_state.copy_to_host()
    print(f"lj256_npt: {time.time() - t0:.1f}s  box={conf.simbox.lengths} ts={ts} bs={bs}")
    np.savez_compressed(
        os.path.join(HERE, "lj256_npt.npz"),
        r0=r0, v0=v0, box0=box, sigma=np.float32(1.0), epsilon=np.float32(1.0), cut=np.float32(2.5),
        temperature=np.float32(T), tau=np.float32(tau), pressure=np.float32(P), tau_p=np.float32(tau_p),
        dt=np.float32(dt), nblist="N squared", skin=np.float32(0.5), blocks=2, steps=8, every=2,
        r=conf["r"], v=conf["v"], r_im=conf.r_im, box=conf.simbox.lengths.copy(), scalars=sim.output["scalars"],
        scalar_names=np.array(sim.output.attrs["scalar_names"]), ts_after_test=ts_test, bs_after_test=bs_test,
        thermostat_state=ts, barostat_state=bs, frames=np.asarray(sim.output["block"]),
        frame_boxes=np.asarray(sim.output["sim_box"]),
    )


CASES = {
    "known_answers": case_known_answers,
    "lj256_sf": case_lj256_sf,
    "lj256_sp": case_lj256_sp,
    "ka1372_cells": case_ka1372_cells,
    "lj256_nve": case_lj256_nve,
    "ka1372_nvt": case_ka1372_nvt,
    "rdf_typed": case_rdf_typed,
    "rdf": case_rdf,
    "sq": case_sq,
    "chain200_bonds": case_chain200_bonds,
    "chain1200_cells": case_chain1200_cells,
    "chain200_nve": case_chain200_nve,
    "lj256_npt": case_lj256_npt,
}

if __name__ == "__main__":
    if sys.argv[1:2] == ["_run"]:
        name = sys.argv[2]
        if name in NO_SIMULATOR:
            _import_gamdpy(simulator=False)
        CASES[name]()
        sys.exit(0)
    # every case in a fresh process: numba reads the simulator switches at import
    for a in sys.argv[1:] or list(CASES):
        subprocess.run([sys.executable, os.path.abspath(__file__), "_run", a], check=True)
