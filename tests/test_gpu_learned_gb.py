"""Learned Born radii in the engine (no reference counterpart; OBC terms from
forces/gbsa_obc.rs:184-309): forces and energy of the learned-radii GB against the f64 oracle
with the same network, the exact-pass judge and online training, what the trained network
gains over the short-range integral alone, and determinism of whole runs."""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu


def gb_only_context(chs, learned=None, precision="mixed", friction=1.0, seed=3):
    sysms = []
    for ch in chs:
        s = ommb200.System()
        gb = ommb200.GBSAOBCForce()
        gb.set_solvent_dielectric(78.5)
        gb.set_solute_dielectric(1.0)
        for q, r in zip(ch.charges, ch.radii):
            s.add_particle(ch.mass)
            gb.add_particle(float(q), float(r), ch.gb_scale)
        if learned is not None:
            gb.set_learned_radii(**learned)
        s.add_force(gb)
        sysms.append(s)
    ctx = ommb200.BatchContext(sysms, systems.langevin(friction=friction, step_size=0.001,
                                                       seed=seed), precision=precision)
    ctx.set_positions(np.concatenate([c.positions for c in chs]))
    return ctx


def chain_context(chs, learned, friction=1.0, seed=3):
    """Full implicit-solvent chains (nonbonded, bonds, angles) with the GBSAOBCForce in force
    group 1."""
    sysms = [systems.chain_system(c, learned_radii=learned, gb_force_group=1) for c in chs]
    ctx = ommb200.BatchContext(sysms, systems.langevin(friction=friction, step_size=0.001,
                                                       seed=seed))
    ctx.set_positions(np.concatenate([c.positions for c in chs]))
    return ctx


def normalised_params(rng, g, target):
    p = np.zeros(O.LR_N_PARAMS, np.float32)
    o = O.LR_OFF
    p[o["W1"]:o["b1"]] = rng.normal(0, 1 / np.sqrt(32), 2048)
    p[o["W2"]:o["b2"]] = rng.normal(0, 1 / np.sqrt(64), 4096)
    p[o["w3"]:o["b3"]] = rng.normal(0, 0.5 / np.sqrt(64), 64)
    p[o["mean"]:o["inv_std"]] = g.mean(0)
    p[o["inv_std"]:o["t_mean"]] = 1 / np.maximum(g.std(0), 1e-3)
    p[o["t_mean"]], p[o["t_scale"]] = target.mean(), target.std()
    return p


def oracle_learned(ch, params):
    g = O.radial_features(ch.positions)
    y, cache = O.mlp_forward(params, g)
    P = O.mlp_unpack(params)
    tail = y * float(P["t_scale"]) + float(P["t_mean"])
    dtail = O.mlp_input_grad(cache) * float(P["t_scale"])
    n = ch.n_atoms
    return O.learned_gbsa(ch.positions, ch.charges, ch.radii, np.full(n, ch.gb_scale), tail,
                          dtail)


@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_learned_forces_and_energy_match_oracle(precision):
    chs = [synth.chain(700, seed=4), synth.chain(300, seed=8)]
    # the network is set by hand (random weights, normalised on these chains) and trusted
    rng = np.random.default_rng(1)
    g = np.concatenate([O.radial_features(c.positions) for c in chs])
    full_short = []
    for c in chs:
        n = c.n_atoms
        _, _, _, short, full = O.learned_gbsa(c.positions, c.charges, c.radii,
                                              np.full(n, c.gb_scale), np.zeros(n),
                                              np.zeros((n, 32)))
        full_short.append(full - short)
    p = normalised_params(rng, g, np.concatenate(full_short))
    ctx = gb_only_context(chs, learned={"judge_interval": 1000}, precision=precision)
    ctx.set_radii_mlp_params(p)
    st = ctx.get_state(forces=True, energy=True)
    pot, _ = ctx.system_energies()
    assert ctx.learned_radii_stats()["active"]
    for k, (c, f) in enumerate(zip(chs, ctx.split(st.forces))):
        f_ref, e_ref, *_ = oracle_learned(c, p)
        err = float(np.sqrt(((f - f_ref) ** 2).sum() / (f_ref ** 2).sum()))
        print(f"chain {k}: force rms rel {err:.2e}, E {pot[k]:.6f} vs {e_ref:.6f}")
        assert err < 2e-4
        assert abs(pot[k] - e_ref) < 2e-5 * abs(e_ref)


def compact_globule(n, seed, spacing=0.3):
    """n particles on a jittered cubic lattice filling a ball: every 32-particle block lies
    within the 2 nm integral cutoff of most others, so a block's neighbour list runs over
    several of the kernels' 16-block chunks."""
    rng = np.random.default_rng(seed)
    m = int(np.ceil((6 * n / np.pi) ** (1 / 3))) + 2
    g = (np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3)
         - (m - 1) / 2) * spacing
    g = g[np.argsort((g ** 2).sum(1), kind="stable")][:n]
    pos = g + rng.uniform(-0.03, 0.03, g.shape)
    q = rng.normal(0.0, 0.3, n)
    return synth.Chain(positions=pos, charges=q - q.mean(), radii=rng.uniform(0.12, 0.2, n))


@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_learned_matches_oracle_when_block_lists_span_chunks(precision):
    chs = [compact_globule(1200, seed=5)]
    nb = (1200 + 31) // 32
    lo = np.array([chs[0].positions[32 * b:32 * b + 32].min(0) for b in range(nb)])
    hi = np.array([chs[0].positions[32 * b:32 * b + 32].max(0) for b in range(nb)])
    c, h = (lo + hi) / 2, (hi - lo) / 2
    gap = np.maximum(np.abs(c[:, None] - c[None]) - h[:, None] - h[None], 0)
    assert ((gap ** 2).sum(-1) < 4.0).sum(1).max() > 32  # more than two chunks of 16 blocks
    rng = np.random.default_rng(2)
    g = O.radial_features(chs[0].positions)
    n = 1200
    _, _, _, short, full = O.learned_gbsa(chs[0].positions, chs[0].charges, chs[0].radii,
                                          np.full(n, chs[0].gb_scale), np.zeros(n),
                                          np.zeros((n, 32)))
    p = normalised_params(rng, g, full - short)
    ctx = gb_only_context(chs, learned={"judge_interval": 1000}, precision=precision)
    ctx.set_radii_mlp_params(p)
    st = ctx.get_state(forces=True, energy=True)
    pot, _ = ctx.system_energies()
    assert ctx.learned_radii_stats()["active"]
    f_ref, e_ref, *_ = oracle_learned(chs[0], p)
    err = float(np.sqrt(((st.forces - f_ref) ** 2).sum() / (f_ref ** 2).sum()))
    print(f"globule: force rms rel {err:.2e}, E {pot[0]:.6f} vs {e_ref:.6f}")
    assert err < 2e-4
    assert abs(pot[0] - e_ref) < 2e-5 * abs(e_ref)


def test_judge_trains_and_the_network_gains_over_short_range_alone():
    chs = [synth.chain(1500, seed=11 + k) for k in range(4)]
    learned = {"judge_interval": 25, "radius_tolerance": 0.01, "train_steps": 40}
    ctx = chain_context(chs, learned, friction=5.0)
    ctx.set_velocities_to_temperature(300.0, seed=5)
    ctx.step(1000)
    stats = ctx.learned_radii_stats()
    print(stats)
    assert stats["judges"] == 1000 // 25
    assert stats["learned_steps"] + stats["exact_steps"] == 1000
    assert stats["active"] and stats["learned_steps"] > 0
    assert stats["last_radius_error"] <= 0.01
    # radii of the trained network vs the exact OBC radii, on the CPU oracle, at the current
    # positions: the network must beat both "no tail" and "constant mean tail"
    params = ctx.get_radii_mlp_params()
    P = O.mlp_unpack(params)
    x = ctx.split(ctx.get_state(positions=True).positions)
    errs = {"network": [], "zero": [], "mean": []}
    for c, pos in zip(chs, x):
        n = c.n_atoms
        g = O.radial_features(pos)
        y, _ = O.mlp_forward(params, g)
        tail = y * float(P["t_scale"]) + float(P["t_mean"])
        _, _, born_exact = O.gbsa_obc(pos, c.charges, c.radii, np.full(n, c.gb_scale),
                                      solvent_dielectric=78.5)
        for name, t in [("network", tail), ("zero", np.zeros(n)),
                        ("mean", np.full(n, float(P["t_mean"])))]:
            _, _, born, _, _ = O.learned_gbsa(pos, c.charges, c.radii, np.full(n, c.gb_scale), t,
                                              np.zeros((n, 32)))
            errs[name].append(np.abs(born / born_exact - 1.0))
    summary = {k: (float(np.concatenate(v).mean()), float(np.concatenate(v).max()))
               for k, v in errs.items()}
    print("radius relative error (mean, max):", summary)
    assert summary["network"][0] < 0.5 * summary["zero"][0]
    assert summary["network"][0] < summary["mean"][0]
    assert summary["network"][1] < summary["zero"][1]


def test_learned_energy_tracks_exact_obc():
    chs = [synth.chain(1200, seed=31 + k) for k in range(3)]
    ctx = chain_context(chs, {"judge_interval": 20, "train_steps": 40}, friction=5.0)
    ctx.set_velocities_to_temperature(300.0, seed=2)
    ctx.step(600)
    assert ctx.learned_radii_stats()["active"]
    x = ctx.get_state(positions=True).positions
    pot, _ = ctx.system_energies(groups=1 << 1)  # the GBSAOBCForce alone
    for k, (c, pos) in enumerate(zip(chs, ctx.split(x))):
        n = c.n_atoms
        _, e_exact, _ = O.gbsa_obc(pos, c.charges, c.radii, np.full(n, c.gb_scale),
                                   solvent_dielectric=78.5)
        per_k = abs(pot[k] - e_exact) / (n / 1000.0)
        print(f"chain {k}: learned {pot[k]:.3f} exact {e_exact:.3f} -> {per_k:.3f} kJ/mol per 1000")
        assert per_k < 0.5


def test_learned_runs_are_bit_identical():
    chs = [synth.chain(500, seed=41), synth.chain(260, seed=42)]
    out = []
    for _ in range(2):
        ctx = chain_context(chs, {"judge_interval": 10, "train_steps": 5}, friction=2.0)
        ctx.set_velocities_to_temperature(300.0, seed=7)
        ctx.step(120)
        st = ctx.get_state(positions=True, velocities=True)
        out.append((st.positions, st.velocities, ctx.get_radii_mlp_params(),
                    ctx.learned_radii_stats()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    assert out[0][3] == out[1][3]
