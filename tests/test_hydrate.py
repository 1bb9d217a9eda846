"""Hydration shell (Molecule::generate_new_hydration with RadialHydration, no culling).

CPU: the oracle (oracle_hydrate, a sequential restatement of RadialHydration.cpp:43-206) against the
reference's own waters in tests/golden/hydrate_* (fresh grids and grids kept across rigid moves,
noise tables and none), the grid axes, and the host-only axes call of the C ABI.
GPU: ausaxs_gpu_hydrate (the round-based device resolver) against the same fixtures and against the
oracle on larger structures, bit for bit; edge cases the C ABI must reject or handle."""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist
from oracle import py as O
from tests.helpers import GOLDEN, load_golden

import glob
import os

CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "hydrate_*.npz")))


def noise_of(g, step):
    seed = int(g["noise_seed"])
    return None if seed < 0 else O.hydrate_noise(26 * len(g[f"atoms{step}"]), seed + step)


def per_body(cands, body_sizes):
    # the reference splits the grid's member list by the bodies' sizes in body order
    # (GridBasedHydration.cpp:66-78), whatever order the moves left the members in
    edges = np.cumsum(body_sizes)
    return np.bincount(np.searchsorted(edges, cands // 26, side="right"), minlength=len(body_sizes))


def replay(g, grid):
    """Drives a hydration grid (oracle or device) through a fixture as the reference's rigid-body loop
    drove its grid: all bodies added, then per move the body removed at its old coordinates and added
    back at the end of the member list; yields (step, waters, candidates) per step."""
    sizes = [int(x) for x in g["body_sizes"]]
    order = list(range(len(sizes)))

    def span(k):
        off = 0
        for b in order:
            if b == k:
                return off, off + sizes[b]
            off += sizes[b]

    grid.add(g["atoms0"], g["ff0"])
    for step in range(int(g["steps"])):
        if step:
            k = int(g["moves"][step - 1])
            lo, hi = span(k)
            grid.remove(g[f"atoms{step - 1}"][lo:hi], g[f"ff{step - 1}"][lo:hi])
            order.remove(k)
            order.append(k)
            lo, hi = span(k)
            np.testing.assert_array_equal(g[f"ff{step}"][lo:hi], g[f"ff{step - 1}"][span_before(g, step, k)])
            grid.add(g[f"atoms{step}"][lo:hi], g[f"ff{step}"][lo:hi])
        out = grid.hydrate(g[f"atoms{step}"], g[f"ff{step}"], noise_of(g, step))
        yield step, out[0], out[1]


def span_before(g, step, k):
    # body k's rows in the previous step's member list (moves append the moved body)
    sizes = [int(x) for x in g["body_sizes"]]
    order = list(range(len(sizes)))
    for m in g["moves"][: step - 1]:
        order.remove(int(m))
        order.append(int(m))
    off = 0
    for b in order:
        if b == k:
            return slice(off, off + sizes[b])
        off += sizes[b]


def test_cases_present():
    assert len(CASES) >= 4 and any(int(load_golden(c)["steps"]) > 1 for c in CASES)


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    g = load_golden(case)
    for step, w, cand in replay(g, O.HydrationGrid(g["axes0"])):
        np.testing.assert_array_equal(w, g[f"waters{step}"], err_msg=f"step {step}")
        np.testing.assert_array_equal(per_body(cand, g["body_sizes"]), g[f"per_body{step}"])


def test_fresh_grid_oracle_is_the_kept_grid_oracle_at_step_0():
    for case in CASES:
        g = load_golden(case)
        w, _ = O.hydrate(g["atoms0"], g["ff0"], g["axes0"], noise_of(g, 0))
        np.testing.assert_array_equal(w, g["waters0"])


@pytest.mark.parametrize("case", CASES)
def test_axes_match_reference(case):
    g = load_golden(case)
    np.testing.assert_array_equal(O.hydrate_axes(g["atoms0"]), g["axes0"])
    np.testing.assert_array_equal(_capi.hydrate_axes(g["atoms0"]), g["axes0"])  # host-only C ABI call


def test_axes_small_and_empty():
    # the running box is an int vector: extents truncate toward zero, and the origin is always inside
    xyz = np.array([[-0.9, 0.4, 2.7], [0.2, -3.99, 0.5]])
    np.testing.assert_array_equal(_capi.hydrate_axes(xyz), O.hydrate_axes(xyz))
    np.testing.assert_array_equal(_capi.hydrate_axes(np.zeros((0, 3))), O.hydrate_axes(np.zeros((0, 3))))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_device_grid_matches_reference(case):
    g = load_golden(case)
    grid = _capi.HydrationGrid(_capi.default_context(), g["axes0"])
    try:
        for step, w, cand in replay(g, grid):
            np.testing.assert_array_equal(w, g[f"waters{step}"], err_msg=f"step {step}")
            np.testing.assert_array_equal(per_body(cand, g["body_sizes"]), g[f"per_body{step}"])
    finally:
        grid.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_device_fresh_grid_matches_reference(case):
    g = load_golden(case)
    w, cand, rounds = _capi.hydrate(_capi.default_context(), g["atoms0"], g["ff0"], g["axes0"], noise_of(g, 0))
    np.testing.assert_array_equal(w, g["waters0"])
    np.testing.assert_array_equal(per_body(cand, g["body_sizes"]), g["per_body0"])
    assert rounds >= 1


@pytest.mark.gpu
def test_device_grid_long_history_matches_oracle():
    # many moves of several bodies on one kept grid: the device's order-free marking against the
    # oracle's atom-by-atom restatement of the reference's conditional marking
    def rotation(axis, angle):
        axis = np.asarray(axis, float) / np.linalg.norm(axis)
        K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
        return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K

    rng = np.random.default_rng(77)
    sizes = [300, 250, 200, 150]
    xyz = [rng.normal(c, 5.0, (n, 3)) for c, n in zip(((0, 0, 0), (15, 0, 0), (0, 16, 0), (0, 0, 17)), sizes)]
    ff = [rng.choice([3, 7, 11, 12], n).astype(np.int32) for n in sizes]
    allx = np.concatenate(xyz)
    axes = O.hydrate_axes(allx)
    dev = _capi.HydrationGrid(_capi.default_context(), axes)
    ora = O.HydrationGrid(axes)
    order = list(range(len(sizes)))
    for grid in (dev, ora):
        grid.add(allx, np.concatenate(ff))
    try:
        for step in range(12):
            if step:
                k = int(rng.integers(len(sizes)))
                R = rotation(rng.normal(size=3), rng.uniform(-0.4, 0.4))
                c = xyz[k].mean(0)
                new = (xyz[k] - c) @ R.T + c + rng.uniform(-3, 3, 3)
                b = np.round(new - axes[:3])
                if np.any(b < 8) or np.any(b >= axes[3:] - 8):  # stay well inside the kept axes
                    new = (xyz[k] - c) @ R.T + c
                for grid in (dev, ora):
                    grid.remove(xyz[k], ff[k])
                    grid.add(new, ff[k])
                xyz[k] = new
                order.remove(k)
                order.append(k)
            members = np.concatenate([xyz[b] for b in order])
            types = np.concatenate([ff[b] for b in order])
            noise = O.hydrate_noise(26 * len(members), 100 + step)
            w, c, _ = dev.hydrate(members, types, noise)
            ow, oc = ora.hydrate(members, types, noise)
            np.testing.assert_array_equal(c, oc, err_msg=f"step {step}")
            np.testing.assert_array_equal(w, ow, err_msg=f"step {step}")
    finally:
        dev.close()


def _globule(seed, n):
    from ausaxs_b200 import synth
    xyz, ff = synth.globule(seed, n)
    return xyz.astype(np.float64), ff.astype(np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("n,noisy", [(4000, False), (20000, True)])
def test_device_matches_oracle_on_globules(n, noisy):
    xyz, ff = _globule(40 + n, n)
    noise = O.hydrate_noise(26 * n, 5) if noisy else None
    w, cand, rounds = _capi.hydrate(_capi.default_context(), xyz, ff, None, noise)
    ow, ocand = O.hydrate(xyz, ff, None, noise)
    assert len(ow) > 0.02 * n
    np.testing.assert_array_equal(cand, ocand)
    np.testing.assert_array_equal(w, ow)


@pytest.mark.gpu
def test_device_tight_axes_take_the_out_of_grid_branches():
    # a grid given by the caller that ends close to the atoms: 3rh / 5rh probes leave it and 1rh
    # probes are clamped, the branches a kept grid reaches after large moves
    xyz, ff = _globule(7, 1500)
    ax = O.hydrate_axes(xyz)
    lo = np.floor(xyz.min(0)) - 4
    hi = np.ceil(xyz.max(0)) + 4
    tight = np.concatenate([lo, hi - lo])
    assert np.all(tight[3:] < ax[3:])
    w, cand, _ = _capi.hydrate(_capi.default_context(), xyz, ff, tight, O.hydrate_noise(26 * len(xyz), 9))
    ow, ocand = O.hydrate(xyz, ff, tight, O.hydrate_noise(26 * len(xyz), 9))
    np.testing.assert_array_equal(cand, ocand)
    np.testing.assert_array_equal(w, ow)


@pytest.mark.gpu
def test_device_seeded_noise_is_reproducible():
    xyz, ff = _globule(8, 3000)
    ctx = _capi.default_context()
    a = _capi.hydrate(ctx, xyz, ff, None, None, seed=12345)
    b = _capi.hydrate(ctx, xyz, ff, None, None, seed=12345)
    c = _capi.hydrate(ctx, xyz, ff, None, None, seed=0)
    np.testing.assert_array_equal(a[0], b[0])
    assert not np.array_equal(a[0], c[0][: len(a[0])]) or len(a[0]) != len(c[0])
    # every water keeps its distance: farther than r_vdw from every atom's cell centre is not
    # required, but its own cell must not be an atom's (the reference's first test)
    ax = O.hydrate_axes(xyz)
    atom_cells = {tuple(x) for x in np.round(xyz - ax[:3]).astype(int)}
    assert not any(tuple(x) in atom_cells for x in np.round(a[0] - ax[:3]).astype(int))


@pytest.mark.gpu
def test_device_edge_cases():
    ctx = _capi.default_context()
    w, cand, rounds = _capi.hydrate(ctx, np.zeros((0, 3)), np.zeros(0, np.int32))
    assert len(w) == 0 and rounds == 0
    one = np.array([[1.0, 2.0, 3.0]])
    w, cand, _ = _capi.hydrate(ctx, one, np.array([3], np.int32))
    ow, ocand = O.hydrate(one, np.array([3], np.int32))
    np.testing.assert_array_equal(w, ow)
    # capacity: the count comes back with the error
    xyz, ff = _globule(9, 800)
    n = _capi.C.c_int64(0)
    out = np.zeros((1, 3))
    rc = _capi.load().ausaxs_gpu_hydrate(ctx.h, _capi.fptr(xyz, _capi.C.c_double), _capi.fptr(ff, _capi.C.c_int32),
                                         len(xyz), None, None, 0, _capi.fptr(out, _capi.C.c_double), 1,
                                         _capi.C.byref(n), None, None)
    assert rc == _capi.ERR_CAPACITY and n.value == len(O.hydrate(xyz, ff)[0])
    # a form-factor type without a radius (EXCLUDED_VOLUME), an atom outside the given axes
    with pytest.raises(_capi.AusaxsError):
        _capi.hydrate(ctx, one, np.array([0], np.int32))
    with pytest.raises(_capi.AusaxsError):
        _capi.hydrate(ctx, one, np.array([3], np.int32), np.array([10.0, 10.0, 10.0, 5, 5, 5]))
    # the context stays usable
    w2, _, _ = _capi.hydrate(ctx, one, np.array([3], np.int32))
    np.testing.assert_array_equal(w2, ow)


@pytest.mark.gpu
def test_molecule_generate_new_hydration():
    xyz, ff = _globule(10, 2000)
    m = hist.Molecule(atoms=xyz, ff_types=ff)
    n = m.generate_new_hydration(noise=O.hydrate_noise(26 * len(xyz), 3))
    ow, _ = O.hydrate(xyz, ff, None, O.hydrate_noise(26 * len(xyz), 3))
    assert n == len(ow)
    np.testing.assert_array_equal(m.waters, ow)
    assert np.all(m.water_weights == hist.WATER_CHARGE)


@pytest.mark.gpu
def test_device_pointer_variant_matches_host_variant():
    import torch
    xyz, ff = _globule(11, 3000)
    ctx = _capi.default_context()
    w, cand, rounds = _capi.hydrate(ctx, xyz, ff)
    surv, r2 = _capi.hydration_stats(ctx)
    assert r2 == rounds and surv >= len(w)
    ax = _capi.hydrate_axes(xyz)
    a, f = torch.from_numpy(xyz).cuda(), torch.from_numpy(ff).cuda()
    out = torch.zeros((len(w) + 10, 3), dtype=torch.float64, device="cuda")
    cd = torch.zeros(len(w) + 10, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    n, r = _capi.hydrate_device(ctx, a, f, len(xyz), ax, out, len(w) + 10, cd)
    assert n == len(w) and r == rounds
    np.testing.assert_array_equal(out[:n].cpu().numpy(), w)
    np.testing.assert_array_equal(cd[:n].cpu().numpy(), cand)
