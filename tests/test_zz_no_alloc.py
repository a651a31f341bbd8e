"""The allocation-free entry point against the Context path, through the C ABI.

ommb200_nonbonded_forces_noalloc serves callers that must not allocate device memory -- code
inside another framework's memory pool, or a plugin that may only use the buffers it is
handed.  Its scratch is one static device array shared
by every call, which keeps the previous call's contents, so the check runs two calls in a row
and compares both with the Context's forces and energy (mixed precision, 5e-6 force RMS; energy
within 1e-6 relative plus 5e-7 kJ/mol per particle of FP32 pair-sum noise).
"""
import ctypes as C

import numpy as np
import pytest

import ommb200

pytestmark = pytest.mark.gpu

FORCE_RMS = 5e-6


def particles(n, seed):
    rng = np.random.default_rng(seed)
    side = int(np.ceil(n ** (1 / 3)))
    idx = np.arange(n)
    grid = np.stack([idx % side, (idx // side) % side, idx // (side * side)], 1)
    pos = (grid + 0.5) * 0.32 + rng.uniform(-0.04, 0.04, size=(n, 3))
    q = rng.normal(0.0, 0.4, n)
    q -= q.mean()
    sigma = rng.uniform(0.25, 0.35, n)
    eps = rng.uniform(0.1, 0.8, n)
    return pos, q, sigma, eps


def context_reference(pos, q, sigma, eps, method, cutoff):
    s = ommb200.System()
    nb = ommb200.NonbondedForce()
    nb.set_nonbonded_method(method)
    nb.set_cutoff_distance(cutoff)
    for qi, si, ei in zip(q, sigma, eps):
        s.add_particle(12.0)
        nb.add_particle(float(qi), float(si), float(ei))
    s.add_force(nb)
    ctx = ommb200.Context(s, ommb200.LangevinMiddleIntegrator(300.0, 1.0, 0.002), precision="mixed")
    ctx.set_positions(pos)
    st = ctx.get_state(forces=True, energy=True)
    return st.forces, st.potential_energy


def near_cutoff_pairs(cutoff, seed):
    """32 isolated pairs (5 nm apart, beyond the cutoff of each other) at squared distances
    within 5e-5 rc^2 of rc^2, half inside and half outside: the exact decision band."""
    rng = np.random.default_rng(seed)
    n_pairs = 32
    delta = rng.uniform(1e-8, 5e-5, n_pairs) * np.where(np.arange(n_pairs) % 2 == 0, 1.0, -1.0)
    r = cutoff * np.sqrt(1.0 + delta)
    pos = np.zeros((2 * n_pairs, 3))
    pos[0::2, 0] = 5.0 * np.arange(n_pairs)
    pos[1::2, 0] = pos[0::2, 0] + r
    pos[:, 1] = rng.uniform(-0.5, 0.5)
    q = rng.normal(0.0, 0.5, 2 * n_pairs)
    sigma = rng.uniform(0.25, 0.35, 2 * n_pairs)
    eps = rng.uniform(0.1, 0.8, 2 * n_pairs)
    return pos, q, sigma, eps


CASES = [("NoCutoff", 1), ("NoCutoff", 33), ("NoCutoff", 1500), ("NoCutoff", 8192),
         ("CutoffNonPeriodic", 1), ("CutoffNonPeriodic", 33), ("CutoffNonPeriodic", 1500),
         ("CutoffNonPeriodic", 8192), ("CutoffNonPeriodic", "near")]


@pytest.mark.parametrize("method,n", CASES)
def test_noalloc_matches_context_on_two_calls(method, n):
    """n = 1 (one padded block, no pair), 33 (a second, nearly empty block), 8,192 (the whole
    static scratch) and pairs straddling the cutoff, against the Context, on two calls."""
    import torch

    cutoff = 1.0
    if n == "near":
        pos, q, sigma, eps = near_cutoff_pairs(cutoff, seed=5)
        n = len(q)
    else:
        pos, q, sigma, eps = particles(n, seed=12)
    f_ref, e_ref = context_reference(pos, q, sigma, eps, method, cutoff)
    dev = torch.device("cuda", 0)
    t = {k: torch.tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
         for k, v in dict(pos=pos, q=q, sigma=sigma, eps=eps).items()}
    out_f = torch.empty((n, 3), dtype=torch.float64, device=dev)
    out_e = torch.empty(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    lib = ommb200.library()
    fn = lib.ommb200_nonbonded_forces_noalloc
    D = C.POINTER(C.c_double)
    fn.argtypes = [C.c_int, D, D, D, D, C.c_int, C.c_double, C.c_double, D, D, C.c_void_p]
    fn.restype = C.c_int

    def ptr(x):
        return C.cast(C.c_void_p(x.data_ptr()), D)

    for call in range(2):
        out_f.fill_(float(1000 + call))  # stale values must not survive
        out_e.fill_(-1.0)
        rc = fn(n, ptr(t["pos"]), ptr(t["q"]), ptr(t["sigma"]), ptr(t["eps"]),
                ommb200.NONBONDED_METHODS[method], cutoff, 78.3, ptr(out_f), ptr(out_e),
                C.c_void_p(stream))
        assert rc == ommb200.OK, lib.ommb200_last_error()
        torch.cuda.synchronize(dev)
        f = out_f.cpu().numpy()
        e = float(out_e.item())
        norm = (f_ref ** 2).sum()
        if norm == 0.0:  # a single particle: no pair at all
            assert not f.any() and e == 0.0 and e_ref == 0.0, (call, e, e_ref)
            continue
        err = float(np.sqrt(((f - f_ref) ** 2).sum() / norm))
        assert err < FORCE_RMS, (call, err)
        # FP32 rounding of every pair energy leaves noise that grows with the particle count;
        # it shows where the net energy is a small difference of large terms (reaction field)
        assert abs(e - e_ref) < 1e-6 * abs(e_ref) + 5e-7 * n, (call, e, e_ref)


def test_noalloc_rejects_more_than_its_static_capacity():
    lib = ommb200.library()
    fn = lib.ommb200_nonbonded_forces_noalloc
    dummy = (C.c_double * 1)()
    D = C.POINTER(C.c_double)
    fn.argtypes = [C.c_int, D, D, D, D, C.c_int, C.c_double, C.c_double, D, D, C.c_void_p]
    fn.restype = C.c_int
    p = C.cast(dummy, D)
    rc = fn(8193, p, p, p, p, 0, 1.0, 78.3, p, p, None)
    assert rc == ommb200.ERR_INVALID_ARG
    assert b"8192" in lib.ommb200_last_error()
