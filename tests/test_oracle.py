"""Pins the f64 CPU oracle against the reference's own known-answer and finite-difference tests.

The reference commits no golden output vectors for this path, so these restated tests (each
citing the reference test it mirrors) are what ties the oracle to the reference's behaviour.
Closed forms from outside the reference pin the PME sum further: a direct Ewald sum and the
Madelung energies of rock salt and cesium chloride.  CPU only.
"""
import math

import numpy as np
import pytest

import oracle as O
from ommb200 import synth

K = 138.93545764438198


# --- known answers (tests/golden/known_answers.json) -------------------------------------
@pytest.mark.parametrize("name", ["coulomb", "lj"])
def test_two_particle_known_answers(known_answers, name):
    c = known_answers[name]  # nonbonded.rs:1457-1494
    f, e = O.nonbonded(c["positions"], c["charge"], c["sigma"], c["epsilon"], c["exceptions"],
                       method=c["method"])
    assert abs(e - c["expected_energy"]) < c["tolerance"]
    assert abs(f[0, 0] - c["expected_force0_x"]) < c["tolerance"]
    assert abs(f[1, 0] - c["expected_force1_x"]) < c["tolerance"]


def test_exclusions_known_answer(known_answers):
    c = known_answers["exclusions"]  # nonbonded.rs:1497-1515
    f, _ = O.nonbonded(c["positions"], c["charge"], c["sigma"], c["epsilon"],
                       [tuple(x) for x in c["exceptions"]], method=c["method"])
    assert np.abs(f[0] - np.array(c["expected_force0"])).max() < c["tolerance"]


def test_newtons_third_law():
    # nonbonded.rs:1518-1533
    f, _ = O.nonbonded([[0, 0, 0], [0.5, 0, 0], [0, 0.7, 0]], [0.5, -0.3, 0.1], [0.3, 0.4, 0.35],
                       [0.5, 0.8, 0.3], method="NoCutoff")
    assert np.abs(f.sum(0)).max() < 1e-10


def test_gbsa_isolated_known_answers(known_answers):
    c = known_answers["gbsa_isolated"]  # tests/gbsa_obc.rs:24-58
    for case in c["cases"]:
        f, e, _ = O.gbsa_obc([case["position"]], [case["charge"]], [case["radius"]], [1.0],
                             solvent_dielectric=case["solvent"], solute_dielectric=case["solute"],
                             surface_area_energy=case["surface"])
        assert abs(e - case["expected_energy"]) < c["tolerance"]
        assert np.all(f == 0.0)


def test_lfmiddle_zero_temperature_known_answer(known_answers):
    c = known_answers["lfmiddle_zero_temperature"]  # tests/integrator_compatibility.rs:38-58
    rc, x, v = O.lfmiddle_step([c["position"]], [c["velocity"]], [c["force"]], [c["mass"]],
                               c["step_size"], c["temperature"], c["friction"], np.zeros((1, 3)))
    assert rc == 0
    assert abs(v[0, 0] - c["expected_velocity_x"]) < c["tolerance"]
    assert abs(x[0, 0] - c["expected_position_x"]) < c["tolerance"]


def test_harmonic_bond_known_answers(known_answers):
    c = known_answers["harmonic_bonds"]  # harmonic_bond.rs:187-208
    f, e = O.harmonic_bonds(c["positions"], [tuple(b) for b in c["bonds"]])
    assert abs(f[0, 1] - c["expected_force0_y"]) < c["tolerance"]
    assert abs(f[2, 0] - c["expected_force2_x"]) < c["tolerance"]
    assert abs(f[1, 0] + f[0, 0] + f[2, 0]) < c["tolerance"]
    assert abs(e - c["expected_energy"]) < c["tolerance"]
    c = known_answers["harmonic_bond_periodic"]  # harmonic_bond.rs:210-228
    _, e = O.harmonic_bonds(c["positions"], [tuple(b) for b in c["bonds"]], use_pbc=True,
                            box=np.array(c["box"]))
    assert abs(e - c["expected_energy"]) < c["tolerance"]


def test_harmonic_angle_known_answers(known_answers):
    c = known_answers["harmonic_angles"]  # harmonic_angle.rs:212-259
    eq = c["equilibrium"]
    f, e = O.harmonic_angles(eq["positions"], [tuple(a) for a in eq["angles"]])
    assert abs(e - eq["expected_energy"]) < eq["energy_tolerance"]
    assert np.abs(f).max() < eq["force_tolerance"]
    d = c["displaced"]
    _, e = O.harmonic_angles(d["positions"], [tuple(a) for a in d["angles"]])
    assert abs(e - d["expected_energy"]) < d["energy_tolerance"]
    cons = c["conservation"]
    f, _ = O.harmonic_angles(cons["positions"], [tuple(a) for a in cons["angles"]])
    assert np.abs(f.sum(0)).max() < cons["force_sum_tolerance"]


def test_philox_known_answer_vectors(known_answers):
    for case in known_answers["philox4x32_10"]:
        assert list(O.philox(case["ctr"], case["key"])) == case["out"]


# --- finite differences -------------------------------------------------------------------
def _fd_check(energy_fn, forces, pos, h, rtol, atol=None):
    pos = np.array(pos, dtype=np.float64)
    for i in range(pos.shape[0]):
        for a in range(3):
            p = pos.copy()
            m = pos.copy()
            p[i, a] += h
            m[i, a] -= h
            num = -(energy_fn(p) - energy_fn(m)) / (2 * h)
            tol = rtol * (1.0 + abs(num)) if atol is None else atol + rtol * abs(num)
            assert abs(num - forces[i, a]) < tol, (i, a, num, forces[i, a])


@pytest.mark.parametrize("method", ["NoCutoff", "CutoffNonPeriodic", "CutoffPeriodic", "PME"])
def test_nonbonded_forces_are_energy_gradients(method):
    # tests/nonbonded_gradients.rs:18-53 (switching on, triclinic box)
    box = np.array([[3.0, 0, 0], [0.4, 3.0, 0], [-0.2, 0.3, 3.0]])
    pos = np.array([[0.1, 0.2, 0.3], [0.9, 0.4, 0.2], [2.8, 0.7, 0.4]])
    kw = dict(method=method, cutoff=1.2, ewald_tolerance=1e-5, box=box, use_switching=True,
              switching_distance=0.8)
    args = ([0.4, -0.3, 0.1], [0.3, 0.32, 0.34], [0.5, 0.6, 0.7], [(0, 2, -0.02, 0.32, 0.4)])
    f, _ = O.nonbonded(pos, *args, **kw)
    _fd_check(lambda p: O.nonbonded(p, *args, **kw)[1], f, pos, 1e-5, 5e-5)


def test_pme_triclinic_reciprocal_gradient():
    # nonbonded.rs:1364-1413 (PME, exceptions with PBC)
    box = np.array([[3.0, 0, 0], [0.3, 3.0, 0], [-0.3, 0.3, 3.0]])
    pos = np.array([[0.1, 0.2, 0.3], [0.6, 0.4, 0.2], [2.8, 0.7, 0.4]])
    kw = dict(method="PME", cutoff=1.2, ewald_tolerance=1e-5, box=box, exceptions_use_pbc=True)
    args = ([0.4, -0.3, 0.1], [0.3, 0.32, 0.34], [0.5, 0.6, 0.7], [(0, 2, -0.02, 0.32, 0.4)])
    f, _ = O.nonbonded(pos, *args, **kw)
    _fd_check(lambda p: O.nonbonded(p, *args, **kw)[1], f, pos, 5e-4, 1e-4, atol=1e-3)


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("surface", [0.0, 2.25936])
def test_gbsa_gradients_with_burial(method, surface):
    # tests/gbsa_obc.rs:61-112
    box = np.array([[2.0, 0, 0], [0.6, 2.1, 0], [-0.4, 0.3, 2.2]])
    pos = np.array([[0.1, 0.2, 0.3], [0.135, 0.225, 0.32], [0.7, 0.4, 0.5], [1.8, 0.2, 0.3]])
    q, r, s = [0.4, -0.3, 0.2, -0.5], [0.3, 0.1, 0.17, 0.13], [1.2, 0.8, 0.7, 0.9]
    kw = dict(method=method, cutoff=0.9, surface_area_energy=surface, box=box)
    f, _, _ = O.gbsa_obc(pos, q, r, s, **kw)
    _fd_check(lambda p: O.gbsa_obc(p, q, r, s, **kw)[1], f, pos, 1e-6, 2e-6)
    assert np.abs(f.sum(0)).max() < 1e-10


# --- pair set (neighbors.rs:184-263) ------------------------------------------------------
def _brute_pairs(pos, cutoff, box):
    pos = np.asarray(pos)
    n = len(pos)
    out = set()
    for i in range(n):
        for j in range(i + 1, n):
            d = pos[j] - pos[i]
            if box is not None:
                for k in (2, 1, 0):
                    s = math.floor(d[k] / box[k][k] + 0.5)
                    d[: k + 1] -= s * np.asarray(box[k][: k + 1])
            if float(d @ d) < cutoff * cutoff:
                out.add((i, j))
    return out


@pytest.mark.parametrize("box", [None, [[2.0, 0, 0], [0.7, 2.0, 0], [-0.4, 0.5, 2.0]],
                                 [[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]]])
@pytest.mark.parametrize("cutoff", [0.2, 0.7, 1.1])
def test_cell_pair_set_matches_brute_force(box, cutoff):
    pos = np.array([(((i * 137 + 37) % 997) / 121.0 - 4.0) for i in range(240)]).reshape(80, 3)
    b = None if box is None else np.array(box)
    got = O.pair_set(pos, cutoff, box=b, use_cells=True)
    got_set = {tuple(p) for p in got.tolist()}
    assert len(got_set) == len(got), "duplicate pair"
    assert got_set == _brute_pairs(pos, cutoff, b)


def test_lattice_pair_set_outer_layer():
    # neighbors.rs:190-223
    for t in ([0, 0, 0], [-4.2, 7.1, -0.3]):
        i = np.arange(1024)
        pos = np.stack([0.3 * (i % 11) + t[0], 0.3 * ((i // 11) % 11) + t[1], 0.3 * (i // 121) + t[2]], 1)
        got = O.pair_set(pos, 0.8, use_cells=True)
        ref = O.pair_set(pos, 0.8, use_cells=False)
        assert {tuple(p) for p in got.tolist()} == {tuple(p) for p in ref.tolist()}


# --- PME against an independent method ----------------------------------------------------
def test_pme_agrees_with_direct_ewald():
    rng = np.random.default_rng(3)
    box = np.array([[2.0, 0, 0], [0.3, 2.1, 0], [-0.2, 0.4, 1.9]])
    pos = rng.random((24, 3)) * 1.9
    q = rng.normal(size=24)
    q -= q.mean()
    alpha, dims = 3.0, (40, 42, 38)
    fp, ep = O.pme_reciprocal(pos, q, box, alpha, dims)
    fe, ee = O.ewald_reciprocal(pos, q, box, alpha, 12)
    assert abs(ep - ee) < 1e-6 * abs(ee)
    assert np.sqrt(((fp - fe) ** 2).sum() / (fe ** 2).sum()) < 1e-5


def _rock_salt(cells, a):
    """Conventional rock-salt cells (4 cation + 4 anion sites each), a cubic periodic box."""
    g = np.arange(2 * cells) * (a / 2)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([x, y, z], -1).reshape(-1, 3) + 0.01
    idx = np.stack(np.meshgrid(*[np.arange(2 * cells)] * 3, indexing="ij"), -1).reshape(-1, 3)
    q = np.where(idx.sum(1) % 2 == 0, 1.0, -1.0)
    return pos, q, np.eye(3) * cells * a


def _cesium_chloride(cells, a):
    """Simple-cubic cations with anions at the cube centres, a cubic periodic box."""
    g = np.arange(cells) * a
    c = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = np.vstack([c, c + a / 2]) + 0.01
    q = np.concatenate([np.ones(len(c)), -np.ones(len(c))])
    return pos, q, np.eye(3) * cells * a


@pytest.mark.parametrize("lattice,cells,a,madelung,r0_per_a", [
    ("rock salt", 4, 0.5628, 1.74756459463, 0.5),
    ("cesium chloride", 5, 0.4123, 1.76267477307, math.sqrt(3) / 2),
])
def test_pme_reproduces_madelung_energies(lattice, cells, a, madelung, r0_per_a):
    """An analytic pin of the whole PME sum (direct, reciprocal and self terms,
    nonbonded.rs:771-1042, pme.rs:141-425): for a neutral ionic crystal whose periodic cell has
    no dipole, the Ewald energy with conducting boundaries is the Madelung lattice energy,
    -(N/2) M k_e q^2 / r0 (r0 the nearest-neighbour distance), and by symmetry no ion feels a
    force."""
    pos, q, box = (_rock_salt if lattice == "rock salt" else _cesium_chloride)(cells, a)
    n = len(q)
    f, e = O.nonbonded(pos, q, np.full(n, 0.1), np.zeros(n), [], method="PME", cutoff=1.0,
                       ewald_tolerance=1e-6, box=box, use_dispersion_correction=False,
                       threads=8)
    exact = -(n / 2) * madelung * K / (r0_per_a * a)
    assert abs(e - exact) < 3e-6 * abs(exact), (e, exact)
    assert np.abs(f).max() < 1e-2  # against pair forces of K / r0^2 ~ 1,700 kJ/mol/nm


@pytest.mark.parametrize("method", ["CutoffNonPeriodic", "CutoffPeriodic"])
def test_reaction_field_pair_closed_form(method):
    """nonbonded.rs:1222-1243: a pair inside the cutoff has E = k q1 q2 (1/r + k_rf r^2 - c_rf)
    with k_rf = (e_rf - 1) / ((2 e_rf + 1) rc^3), c_rf = 3 e_rf / ((2 e_rf + 1) rc), and the
    force along the pair k q1 q2 (1/r^2 - 2 k_rf r)."""
    r, rc, e_rf, q1, q2 = 0.5, 1.0, 78.3, 0.7, -0.4
    kw = dict(method=method, cutoff=rc, reaction_field_dielectric=e_rf,
              use_dispersion_correction=False)
    if method == "CutoffPeriodic":
        kw["box"] = np.eye(3) * 3.0
    f, e = O.nonbonded([[0, 0, 0], [r, 0, 0]], [q1, q2], [0.1, 0.1], [0, 0], [], **kw)
    krf = (e_rf - 1) / ((2 * e_rf + 1) * rc**3)
    crf = 3 * e_rf / ((2 * e_rf + 1) * rc)
    assert abs(e - K * q1 * q2 * (1 / r + krf * r * r - crf)) < 1e-12
    assert abs(f[1, 0] - K * q1 * q2 * (1 / r**2 - 2 * krf * r)) < 1e-11
    assert abs(f[0, 0] + f[1, 0]) < 1e-12


@pytest.mark.parametrize("r", [0.85, 0.95])
def test_lj_switching_closed_form(r):
    """nonbonded.rs:888-900: between the switching distance and the cutoff the LJ energy is
    multiplied by S(t) = 1 - 10 t^3 + 15 t^4 - 6 t^5, t = (r - rs) / (rc - rs), and the force is
    -(dU/dr S + U dS/dr)."""
    sig, eps, rs, rc = 0.3, 0.6, 0.8, 1.0
    f, e = O.nonbonded([[0, 0, 0], [r, 0, 0]], [0, 0], [sig, sig], [eps, eps], [],
                       method="CutoffNonPeriodic", cutoff=rc, use_switching=True,
                       switching_distance=rs, use_dispersion_correction=False)
    t = (r - rs) / (rc - rs)
    s = 1 - 10 * t**3 + 15 * t**4 - 6 * t**5
    ds = (-30 * t**2 + 60 * t**3 - 30 * t**4) / (rc - rs)
    sr6 = (sig / r) ** 6
    u = 4 * eps * (sr6 * sr6 - sr6)
    du = 4 * eps * (-12 * sr6 * sr6 + 6 * sr6) / r
    assert abs(e - u * s) < 1e-15
    assert abs(f[1, 0] + (du * s + u * ds)) < 1e-14


def test_direct_and_reciprocal_parts_sum_to_the_whole():
    """tests/force_groups.rs:55-96 (the PME case): the direct-space part and the
    reciprocal-space part (each with the corrections it owns) add up to the complete
    NonbondedForce, energies to 1e-10 and forces to rounding."""
    pos = [[0.1, 0.2, 0.3], [0.6, 0.4, 0.2], [2.8, 0.7, 0.4]]
    args = (pos, [0.4, -0.3, 0.1], [0.3, 0.32, 0.34], [0.5, 0.6, 0.7],
            [(0, 2, -0.02, 0.32, 0.4)])
    kw = dict(method="PME", cutoff=1.0, box=np.eye(3) * 3.0)
    f_all, e_all = O.nonbonded(*args, **kw)
    f_dir, e_dir = O.nonbonded(*args, include_reciprocal=False, **kw)
    f_rec, e_rec = O.nonbonded(*args, include_direct=False, **kw)
    assert abs(e_all - e_dir - e_rec) < 1e-10
    assert np.abs(f_all - f_dir - f_rec).max() < 1e-10
    assert e_dir != 0.0 and e_rec != 0.0


def test_dispersion_correction_is_the_lj_tail_integral():
    """nonbonded.rs:660-719 for identical particles: the correction is the LJ energy beyond the
    cutoff of a uniform fluid, (N^2 / 2V) int_rc^inf 4 pi r^2 4 eps [(s/r)^12 - (s/r)^6] dr =
    8 pi N^2 eps / V [s^12 / (9 rc^9) - s^6 / (3 rc^3)], whatever the positions."""
    box_len, n_side, sig, eps, rc = 3.0, 5, 0.3, 0.5, 1.0
    g = (np.arange(n_side) + 0.5) * box_len / n_side
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    n = len(pos)
    args = (pos, np.zeros(n), np.full(n, sig), np.full(n, eps), [])
    kw = dict(method="CutoffPeriodic", cutoff=rc, box=np.eye(3) * box_len)
    _, with_tail = O.nonbonded(*args, use_dispersion_correction=True, **kw)
    _, without = O.nonbonded(*args, use_dispersion_correction=False, **kw)
    tail = 8 * math.pi * n * n * eps / box_len**3 * (sig**12 / (9 * rc**9) - sig**6 / (3 * rc**3))
    assert abs((with_tail - without) - tail) < 1e-12 * abs(tail)


# --- virial = -dU/d(strain) ---------------------------------------------------------------
def test_virial_matches_strain_derivative():
    w = synth.water_box(40, 1.9, (4, 4, 3), seed=5)
    args = (w.charges(), w.sigmas(), w.epsilons(), w.exceptions())
    kw = dict(method="PME", cutoff=0.9, ewald_tolerance=1e-5, box=w.box, pme=(3.3, (24, 24, 24)))
    _, _, vir = O.nonbonded(w.positions, *args, virial=True, **kw)
    h = 1e-6
    assert np.abs(vir - vir.T).max() < 1e-9 * np.abs(vir).max()
    # strains with b >= a keep the box in the reduced form the minimum image assumes
    for a in range(3):
        for b in range(a, 3):
            e = []
            for sgn in (1, -1):
                eps = np.zeros((3, 3))
                eps[a, b] = sgn * h
                t = np.eye(3) + eps
                e.append(O.nonbonded(w.positions @ t.T, *args, **{**kw, "box": w.box @ t.T})[1])
            num = -(e[0] - e[1]) / (2 * h)
            assert abs(num - vir[a, b]) < 2e-3 * (1 + abs(num)), (a, b, num, vir[a, b])


# --- constraints and integration ----------------------------------------------------------
WATER = dict(masses=[16.0, 1.0, 1.0], cons=[(0, 1, 0.1), (0, 2, 0.1), (1, 2, 0.16)],
             pos=[[0.0, 0.0, 0.0], [0.08, 0.06, 0.0], [-0.08, 0.06, 0.0]])


def test_constraint_projection_preserves_center_of_mass():
    # tests/constraints.rs:15-39
    m = [1.0, 2.0]
    rc, x = O.constraints_solve([(0, 1, 1.0)], m, [[0, 0, 0], [1.2, 0, 0]], [[0, 0, 0], [1.2, 0, 0]],
                                False, 1e-6)
    assert rc == 0
    assert abs(x[1, 0] - x[0, 0] - 1.0) < 2e-6 and abs(x[0, 0] + 2 * x[1, 0] - 2.4) < 2e-6
    rc, v = O.constraints_solve([(0, 1, 1.0)], m, x, [[1, 2, 0], [-1, -1, 0]], True, 1e-6)
    assert rc == 0
    assert abs(v[1, 0] - v[0, 0]) < 2e-6 and abs(v[0, 0] + 2 * v[1, 0] + 1.0) < 2e-6
    assert v[0, 1] == 2.0 and v[1, 1] == -1.0


@pytest.mark.parametrize("mode", [0, 1])
def test_rigid_water_preserved_by_lfmiddle(mode):
    # tests/constraints.rs:41-76 (LangevinMiddle 300 K, 2/ps, 1 fs, 100 steps)
    x = np.array(WATER["pos"])
    v = np.array([[0.2, 0.1, 0.0]] * 3)
    for step in range(100):
        noise = O.gaussian_noise(11, 0, step, 3)
        rc, x, v = O.lfmiddle_step(x, v, np.zeros((3, 3)), WATER["masses"], 0.001, 300.0, 2.0, noise,
                                   constraints=WATER["cons"], tolerance=1e-5, mode=mode,
                                   waters=[[0, 1, 2]], d_oh=0.1, d_hh=0.16)
        assert rc == 0
        for i, j, d in WATER["cons"]:
            assert abs(np.linalg.norm(x[i] - x[j]) / d - 1.0) < 2e-5


def test_singular_projection_returns_error():
    # tests/constraints.rs:77-97
    rc, x = O.constraints_solve([(0, 1, 1.0)], [1.0, 1.0], np.zeros((2, 3)), np.zeros((2, 3)), False, 1e-5)
    assert rc == -2


def test_settle_equals_converged_shake():
    w = synth.water_box(27, 1.0, (3, 3, 3), seed=9)
    rng = np.random.default_rng(1)
    ref = w.positions
    new = ref + rng.normal(scale=0.004, size=ref.shape)
    rc1, xs = O.settle_positions(w.waters(), synth.D_OH, synth.D_HH, w.masses(), ref, new)
    rc2, xk = O.constraints_solve(w.constraints(), w.masses(), ref, new, False, 1e-13)
    assert rc1 == 0 and rc2 == 0
    assert np.abs(xs - xk).max() < 1e-11
    vel = rng.normal(size=ref.shape)
    rc1, vs = O.settle_velocities(w.waters(), w.masses(), xs, vel)
    rc2, vk = O.constraints_solve(w.constraints(), w.masses(), xs, vel, True, 1e-14)
    assert rc1 == 0 and rc2 == 0
    assert np.abs(vs - vk).max() < 1e-9


def test_massless_particles_remain_fixed():
    # tests/integrator_compatibility.rs:13-36
    x = np.array([[1.0, 2.0, 3.0], [0.0, 0.0, 0.0]])
    v = np.array([[4.0, 5.0, 6.0], [0.1, 0.2, 0.3]])
    f = np.array([[8.0, 9.0, 10.0], [0.1, 0.2, 0.3]])
    for step in range(10):
        rc, x, v = O.lfmiddle_step(x, v, f, [0.0, 2.0], 0.01, 300.0, 2.0, O.gaussian_noise(3, 0, step, 2))
    assert list(x[0]) == [1.0, 2.0, 3.0] and list(v[0]) == [4.0, 5.0, 6.0]
    assert np.isfinite(x).all() and np.isfinite(v).all()


def test_equipartition_free_particles():
    # langevin.rs:289-331: 32 particles of 12 Da, 300 K, friction 3/ps, 10 fs
    n, m = 32, 12.0
    x = np.zeros((n, 3))
    v = np.zeros((n, 3))
    f = np.zeros((n, 3))
    masses = [m] * n
    ek = 0.0
    for step in range(7000):
        rc, x, v = O.lfmiddle_step(x, v, f, masses, 0.01, 300.0, 3.0, O.gaussian_noise(21, 0, step, n))
        if step >= 5000:
            ek += O.kinetic_energy(v, masses)
    kb = 1.380649e-23 * 6.02214076e23 / 1000.0
    expected = 0.5 * 3 * n * kb * 300.0
    assert abs(ek / 2000 - expected) < 0.12 * expected


def test_lfmiddle_one_step_variances_and_moments():
    """tests/stochastic.rs:173-216 for LangevinMiddle: from rest with no force, one step gives
    velocities of variance kT/m (1 - exp(-2 gamma dt)) for each mass, positions v dt/2
    exactly, and normalized velocities with the Gaussian moments 0, 1, 3 (within six standard
    errors)."""
    count, temperature, friction, dt = 60000, 310.0, 2.1, 0.003
    masses = np.array([[1.0, 4.0, 9.0][i % 3] for i in range(count)])
    zero = np.zeros((count, 3))
    rc, x, v = O.lfmiddle_step(zero, zero, zero, masses, dt, temperature, friction,
                               O.gaussian_noise(371, 0, 0, count))
    assert rc == 0
    assert np.abs(x - v * dt / 2).max() < 1e-15
    kb = 1.380649e-23 * 6.02214076e23 / 1000.0
    for group in range(3):
        var = kb * temperature / masses[group] * -np.expm1(-2.0 * friction * dt)
        z = (v[group::3] / np.sqrt(var)).reshape(-1)
        for moment, target, spread in [(1, 0.0, 1.0), (2, 1.0, 2.0), (4, 3.0, 96.0)]:
            assert abs((z ** moment).mean() - target) < 6.0 * np.sqrt(spread / z.size), moment


def test_gaussian_stream_moments():
    z = O.gaussian_noise(123, 0, 7, 200000).reshape(-1)
    assert abs(z.mean()) < 0.01
    assert abs(z.var() - 1.0) < 0.01
    assert abs((z ** 4).mean() - 3.0) < 0.05


def test_water_box_pme_parameters_follow_tolerance_rule():
    # nonbonded.rs:647-658 on the three water boxes
    for name, grid in [("water-1944", 25), ("water-23958", 56)]:
        w = synth.water_preset(name)
        alpha, dims = O.pme_parameters(0.9, 5e-4, w.box)
        assert abs(alpha - 2.92029) < 1e-5 and dims == (grid,) * 3
    alpha, dims = O.pme_parameters(0.9, 5e-4, np.diag([22.0] * 3))
    assert dims == (196,) * 3


def test_barostat_restatement():
    # system.rs:100-141: union-find over constraints and bonds, smaller root
    assert O.molecules(6, constraints=[(4, 5)], bonds=[(2, 0), (3, 4)]) == [[0, 2], [1], [3, 4, 5]]
    # context.rs:976-1028: rigid moves shift molecules by their centroid, others scale points
    pos = np.array([[0.2, 0.3, 0.4], [0.9, 0.3, 0.4], [1.4, 1.1, 0.8]])
    r = O.scale_positions(pos, [[0, 1], [2]], 1.1, True)
    assert np.allclose(r[1] - r[0], pos[1] - pos[0], atol=1e-15)
    assert np.allclose(r[2], 1.1 * pos[2], atol=1e-15)
    assert np.allclose(O.scale_positions(pos, [[0, 1], [2]], 1.1, False), 1.1 * pos)
    # barostat.rs:144-160
    kt = O.BOLTZMANN * 300.0
    w = O.barostat_work(1.0, 1.0, 10.0, 10.1, 5, 300.0)
    assert abs(w - (1.0 + O.BAR_NM3_TO_KJ_PER_MOL * 0.1 - 5 * kt * np.log(1.01))) < 1e-15
    assert O.barostat_accepts(-1.0, 300.0, 0.99) and not O.barostat_accepts(np.nan, 300.0, 0.0)
    assert O.barostat_accepts(kt, 300.0, np.exp(-1.0) - 1e-12)
    assert not O.barostat_accepts(kt, 300.0, np.exp(-1.0) + 1e-12)
    assert not O.barostat_accepts(1.0, 0.0, 0.0)
    # barostat.rs:172-189: 10 rejections shrink the step by 1.1, 10 acceptances grow it
    s = O.VolumeStep(100.0)
    for _ in range(10):
        s.record(False, 100.0)
    assert abs(s.scale - 1.0 / 1.1) < 1e-15 and s.attempted == 0
    for _ in range(10):
        s.record(True, 100.0)
    assert abs(s.scale - 1.0) < 1e-15
