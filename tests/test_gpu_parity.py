"""GPU parity: the sm_100a path (through the C ABI) against the CPU oracle
on the same inputs.  Integer/index outputs are bit-exact; with
exact_math=1 the float outputs are bit-exact too; the default (contracted)
arithmetic is held to the reference's own bars (CheckCuda.cu)."""
import numpy as np
import pytest

from conftest import bits, rel_err, same_bits

pytestmark = pytest.mark.gpu


def with_central_contacts(state, count=8):
    """Small bodies placed overlapping the heaviest body at spread angles and
    varied velocities (withCentralContacts, CheckCuda.cu:198-227)."""
    s = state.copy()
    c = int(np.argmax(s["radius"]))
    n = len(s)
    for k in range(count):
        i = (k + 1) * n // (count + 1)
        if i == c:
            i += 1
        ang = np.float32(6.2831853 * k / count)
        d = np.array([np.cos(ang), np.sin(ang)], np.float32)
        depth = np.float32(0.2 + 0.1 * k)
        pos = np.array([s["px"][c], s["py"][c]], np.float32) + d * (
            s["radius"][c] + s["radius"][i] - depth)
        t = np.array([-d[1], d[0]], np.float32)
        v = [d * -5.0, d * 3.0, t * 4.0][k % 3]
        s["px"][i], s["py"][i] = pos
        s["vx"][i] = s["vx"][c] + v[0]
        s["vy"][i] = s["vy"][c] + v[1]
    return s


def gpu_build(nbx, bodies, **kw):
    sim = nbx.Simulation(bodies, **kw)
    sim.phase("build")
    return sim


STATES = {}


def state(nbx, oracle, name):
    if name in STATES:
        return STATES[name]
    if name == "disc10k":
        s = nbx.uniform_disc(10000)
    elif name == "disc200k":
        s = nbx.uniform_disc(200000)
    elif name == "two_discs65k":
        s = nbx.two_discs(65536, 0, 0.2)
    elif name == "cold50k":
        s = nbx.cold_square(50000, 1)
    elif name == "colliding20k":
        sim = nbx.Simulation(nbx.uniform_disc(20000))
        sim.step(300)
        sim.phase("iterate")
        s = sim.download()
        sim.close()
    elif name == "clumped":
        # tight clumps inside depth-16 Morton cells: runs of equal high code
        # bits of 17 to ~3000 bodies with distinct low bits
        s = nbx.uniform_disc(20000)
        rng = np.random.default_rng(3)
        for start, count, cx, cy, size in ((100, 17, 3.0, -2.0, 1e-3),
                                           (2000, 500, 10.0, 5.0, 1e-2),
                                           (5000, 3000, -20.0, 30.0, 1.5e-2)):
            sl = slice(start, start + count)
            s["px"][sl] = (cx + rng.uniform(-size, size, count)).astype(np.float32)
            s["py"][sl] = (cy + rng.uniform(-size, size, count)).astype(np.float32)
    elif name == "coincident":
        s = nbx.uniform_disc(3000)
        s["px"][100:160] = s["px"][100]  # 60 bodies on one point: depth-32 leaf
        s["py"][100:160] = s["py"][100]
    else:
        raise KeyError(name)
    STATES[name] = s
    return s


@pytest.mark.parametrize("name", ["disc10k", "disc200k", "two_discs65k",
                                  "cold50k", "coincident", "clumped"])
@pytest.mark.parametrize("leaf", [16, 4])
def test_morton_perm_tree_bit_exact(nbx, oracle, name, leaf):
    b = state(nbx, oracle, name)
    sim = gpu_build(nbx, b, leaf_capacity=leaf)
    codes, perm = sim.morton()
    root, ocodes, operm, sb, tree = oracle.morton_build(b, leaf)
    assert np.array_equal(codes, ocodes)
    assert np.array_equal(perm, operm)
    t = sim.tree()
    assert t["node_count"] == tree.node_count
    assert t["level_count"] == tree.level_count
    for k, v in tree.trimmed().items():
        assert same_bits(t[k], v), k
    # the device state is permuted into Morton order like the reference's
    assert np.array_equal(sim.download()["id"], sb["id"])
    sim.close()


@pytest.mark.parametrize("name", ["disc10k", "disc200k", "colliding20k", "cold50k",
                                  "clumped"])
@pytest.mark.parametrize("theta", [1.0, 0.5])
def test_forces(nbx, oracle, name, theta):
    b = state(nbx, oracle, name)
    _, _, _, sb, tree = oracle.morton_build(b)
    ox, oy = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, theta, 1.0)
    sim = nbx.Simulation(b, theta=theta, exact_math=1)
    sim.phase("attract")
    g = sim.download()
    # exact arithmetic: bit-identical to the reference traversal
    assert same_bits(g["ax"], ox) and same_bits(g["ay"], oy)
    sim.set_params(exact_math=0)
    sim.phase("forces")
    g = sim.download()
    e = rel_err(g["ax"], g["ay"], ox, oy)
    assert np.percentile(e, 99) < 1e-5 and e.max() < 1e-4, (np.percentile(e, 99), e.max())
    sim.close()


@pytest.mark.parametrize("name", ["disc10k", "colliding20k"])
def test_forces_vs_partition_quadtree(nbx, oracle, name):
    """Against QuadTree.cpp's own tree (partition build): the bar of
    CheckCuda.cu:609-614 (median < 1e-5, p99 < 1e-4)."""
    b = state(nbx, oracle, name)
    q = np.sort(oracle.quadtree_forces(b, 1.0, 1.0), order="id")
    sim = nbx.Simulation(b)
    sim.phase("attract")
    g = np.sort(sim.download(), order="id")
    e = rel_err(g["ax"], g["ay"], q["ax"], q["ay"])
    assert np.median(e) < 1e-5 and np.percentile(e, 99) < 1e-4
    sim.close()


def collide_cases(nbx, oracle, golden):
    yield "golden", golden["collide_in"]
    c20 = state(nbx, oracle, "colliding20k")
    yield "colliding20k", c20
    yield "central8", with_central_contacts(c20, 8)
    big = nbx.uniform_disc(200000)
    yield "central8_200k", with_central_contacts(oracle.integrate(big, 0.05), 8)
    cold = nbx.cold_square(20000, 2)
    cold["px"] *= np.float32(0.35)  # compressed: most boxes overlap neighbours
    cold["py"] *= np.float32(0.35)
    yield "cold_dense", cold


def test_collisions_bit_exact(nbx, oracle, golden):
    seen_large = 0
    for label, st in collide_cases(nbx, oracle, golden):
        sim = nbx.Simulation(st)
        sim.phase("collide")
        gl, ge = sim.pairs()
        ol, oe = oracle.collision_pairs(st)
        assert len(ol) > 0, label
        assert np.array_equal(gl, ol) and np.array_equal(ge, oe), label
        out = sim.download()
        ref, _ = oracle.collide(st)
        assert same_bits(out, ref), (label, int((out != ref).sum()))
        heavy = int(np.argmax(st["radius"]))
        seen_large += int(((gl == heavy) | (ge == heavy)).sum())
        sim.close()
    assert seen_large > 0  # the large-body path saw real contacts


def test_collision_stats(nbx, oracle):
    """Pair count and the longest chain of dependent pairs (each pair waits
    for the last earlier pair sharing a body) from the oracle's pair list."""
    st = state(nbx, oracle, "colliding20k")
    sim = nbx.Simulation(with_central_contacts(st, 8))
    sim.phase("collide")
    pairs, depth = sim.collision_stats()
    ol, oe = oracle.collision_pairs(with_central_contacts(st, 8))
    last = {}
    deepest = 0
    for a, b in zip(ol.tolist(), oe.tolist()):
        d = max(last.get(a, 0), last.get(b, 0)) + 1
        last[a] = last[b] = d
        deepest = max(deepest, d)
    assert pairs == len(ol) and depth == deepest and depth >= 2
    sim.close()


def test_collide_then_reference_bodies(nbx, golden):
    """Against the reference's own collide() output (fixture)."""
    sim = nbx.Simulation(golden["collide_in"])
    sim.phase("collide")
    assert same_bits(sim.download(), golden["collide_out"])
    sim.close()


@pytest.mark.parametrize("theta", [1.0, 0.5])
def test_ten_step_trajectories(nbx, oracle, golden, theta):
    b = nbx.uniform_disc(20000)
    o = oracle.step(b, steps=10, theta=theta)
    sim = nbx.Simulation(b, theta=theta, exact_math=1)
    sim.step(10)
    sim.sync()
    assert same_bits(sim.download(), o)  # whole state, bit for bit
    sim.close()
    sim = nbx.Simulation(b, theta=theta)
    sim.step(10)
    sim.sync()
    g = np.sort(sim.download(), order="id")
    r = np.sort(o, order="id")
    e = rel_err(g["px"], g["py"], r["px"], r["py"])
    assert e.max() < 1e-3 and np.median(e) < 1e-5, (e.max(), np.median(e))
    sim.close()
    # against the reference's own Simulation::step (partition tree)
    sim = nbx.Simulation(golden["sim_in"], theta=theta)
    sim.step(10)
    g = sim.download(id_order=True)
    r = np.sort(golden[f"sim10_t{theta}"], order="id")
    e = rel_err(g["px"], g["py"], r["px"], r["py"])
    assert e.max() < 1e-3 and np.median(e) < 1e-4, (e.max(), np.median(e))
    sim.close()


def test_step_timed_same_state(nbx):
    """The timed step graph (event records around the force launch) gives
    the same trajectory as the plain one and one duration per step."""
    b = nbx.two_discs(65536, 0, 0.2)
    a = nbx.Simulation(b, theta=0.5)
    a.step(7)
    ra = a.download()
    a.close()
    t = nbx.Simulation(b, theta=0.5)
    t.step_timed(4)
    t.step(1)
    t.step_timed(2)
    ms = t.force_times(2)
    assert ms.shape == (2,) and (ms > 0).all() and (ms < 1e3).all()
    assert same_bits(t.download(), ra)
    with pytest.raises(nbx.NbxError):
        t.force_times(3)  # only 2 steps in the last timed call
    t.set_params(theta=0.7)  # new graphs; timing still works
    t.step_timed(3)
    assert (t.force_times(3) > 0).all()
    t.close()


@pytest.mark.parametrize("n", [1000, 65536 + 17, 300001])
def test_step_io_equals_upload_step_download(nbx, n):
    """nbx_step_io (the drop-in Simulation::step on host bodies) gives the
    bodies that upload + step + download give, bit for bit: into pinned
    memory (force ranges copied while later ranges compute; 1, 1 and 4
    ranges at these sizes), into pageable memory, in place, and after a
    parameter change (new graphs)."""
    import torch

    b = nbx.two_discs(n, 0, 0.2)
    ref = nbx.Simulation(b, theta=0.5)
    cur = b.copy()
    expect = []
    for k in range(4):
        if k == 2:
            ref.set_params(theta=0.7)
        ref.upload(cur)
        ref.step(1)
        cur = ref.download()
        expect.append(cur)
    ref.close()
    pinned = torch.empty(n * 36, dtype=torch.uint8, pin_memory=True)
    hb = pinned.numpy().view(nbx.BODY_DTYPE)
    sim = nbx.Simulation(b, theta=0.5)
    hb[:] = b
    for k in range(4):
        if k == 2:
            sim.set_params(theta=0.7)
        if k == 1:  # pageable in, pageable out
            out = sim.step_io(hb.copy())
            hb[:] = out
        else:  # pinned, in place
            sim.step_io_ptr(pinned.data_ptr(), pinned.data_ptr(), n)
        assert same_bits(hb, expect[k]), k
    sim.close()


def test_deterministic(nbx):
    b = nbx.uniform_disc(20000)
    outs = []
    for _ in range(2):
        sim = nbx.Simulation(b)
        sim.step(50)
        outs.append(sim.download())
        sim.close()
    assert same_bits(outs[0], outs[1])


def test_tree_invariants_1m(nbx):
    """Size-independent properties at the headline size (1,048,576 bodies)."""
    b = nbx.two_discs(1 << 20, 0, 0.2)
    sim = nbx.Simulation(b, theta=0.5)
    sim.step(3)
    sim.phase("build")
    t = sim.tree()
    s = sim.download()
    n = len(b)
    assert np.array_equal(np.sort(s["id"]), np.arange(n))
    assert abs(float(t["mass"][0]) - float(s["mass"].astype(np.float64).sum())) <= 1e-5 * s["mass"].sum()
    leaf = t["children"] == 0
    st, en = t["start"][leaf], t["end"][leaf]
    order = np.lexsort((en, st))  # empty leaves (s, s) sort before (s, e)
    st, en = st[order], en[order]
    assert st[0] == 0 and en[-1] == n and np.array_equal(st[1:], en[:-1])
    assert (en - st).max() <= 16
    half = (t["size"][leaf] * 0.5 * 1.0001 + 1e-3)[order]
    cx, cy = t["centerX"][leaf][order], t["centerY"][leaf][order]
    owner = np.repeat(np.arange(len(st)), en - st)
    assert np.all(np.abs(s["px"] - cx[owner]) <= half[owner])
    assert np.all(np.abs(s["py"] - cy[owner]) <= half[owner])
    sim.close()


def test_fp64_direct_and_energy(nbx, oracle):
    b = nbx.uniform_disc(20000)
    sim = nbx.Simulation(b)
    sim.step(2)
    s = sim.download()
    rng = np.random.default_rng(5)
    tg = rng.choice(len(b), 256, replace=False).astype(np.uint32)
    gx, gy = sim.direct_fp64(tg)
    ox, oy = oracle.direct_fp64(s, 1.0, tg)
    assert np.max(rel_err(gx, gy, ox, oy)) < 1e-12
    stats, err = sim.force_error(tg)
    acc = s[tg]
    e = rel_err(acc["ax"], acc["ay"], ox, oy)
    assert np.allclose(np.sort(err), np.sort(e), rtol=1e-6, atol=1e-12)
    em = sim.energy_momentum()
    oem = oracle.energy_momentum(s)
    assert np.allclose(em, oem, rtol=1e-12, atol=1e-9)
    sim.close()


def _pair_potential(s, eps, plummer=False):
    """FP64 pairwise potential in numpy (test-side restatement)."""
    x = s["px"].astype(np.float64)
    y = s["py"].astype(np.float64)
    m = s["mass"].astype(np.float64)
    dx = x[None, :] - x[:, None]
    dy = y[None, :] - y[:, None]
    r2 = dx * dx + dy * dy
    np.fill_diagonal(r2, np.inf)
    r = np.sqrt(r2)
    if plummer:
        g = 1.0 / np.sqrt(r2 + eps * eps)
    elif eps > 0:
        g = np.arctan2(eps, r) / eps
    else:
        g = 1.0 / r
    phi = -(g * m[None, :]).sum(axis=1)
    return 0.5 * float(np.sum(m * phi)), phi


def test_fp64_potential(nbx, oracle):
    """The potential of the tree law (and of the Plummer law) in FP64:
    exact over all pairs against the oracle's compensated pair sum, per
    target against a numpy pair sum, the sampled estimate with every body
    sampled equal to the exact one, instances summed separately."""
    b = nbx.uniform_disc(3000)
    sim = nbx.Simulation(b)
    sim.step(2)
    s = sim.download()
    u = sim.potential()
    ou = oracle.potential(s, 1.0)
    assert abs(u - ou) <= 1e-11 * abs(ou), (u, ou)
    est, phi = sim.potential(np.arange(len(s), dtype=np.uint32))
    assert abs(est - u) <= 1e-12 * abs(u)
    nu, nphi = _pair_potential(s, 1.0)
    assert np.max(np.abs(phi - nphi) / np.abs(nphi)) < 1e-11
    tg = np.array([0, 7, 2999, 1500], np.uint32)
    est4, phi4 = sim.potential(tg)
    assert np.array_equal(phi4, phi[tg])
    assert abs(est4 - 0.5 * len(s) / 4 * np.sum(s["mass"][tg] * phi4)) <= 1e-12 * abs(est4)
    sim.close()
    # two instances: pairs only within each
    parts = [nbx.uniform_disc(700, 0), nbx.uniform_disc(500, 3)]
    h = nbx.Handle([700, 500])
    h.upload(np.concatenate(parts))
    u2 = h.potential()
    ref = oracle.potential(parts[0], 1.0) + oracle.potential(parts[1], 1.0)
    assert abs(u2 - ref) <= 1e-11 * abs(ref)
    h.close()
    # Plummer law (force_law 1) and the unsoftened tree law
    for kw, eps, pl in ((dict(force_law=1), 1.0, True), (dict(epsilon=0.0), 0.0, False)):
        sm = nbx.Simulation(nbx.uniform_disc(400), **kw)
        st = sm.download()
        assert abs(sm.potential() - _pair_potential(st, eps, pl)[0]) <= 1e-11 * abs(
            _pair_potential(st, eps, pl)[0])
        sm.close()


def test_id_order_download(nbx):
    b = nbx.uniform_disc(5000)
    sim = nbx.Simulation(b)
    sim.step(3)
    a = sim.download()
    o = sim.download(id_order=True)
    assert np.array_equal(o["id"], np.arange(5000))
    assert same_bits(np.sort(a, order="id"), o)
    sim.close()


@pytest.mark.parametrize("n", [1, 2, 16, 17, 33])
def test_small_sizes(nbx, oracle, n):
    b = nbx.uniform_disc(n)
    sim = nbx.Simulation(b, exact_math=1)
    sim.step(3)
    sim.sync()
    assert same_bits(sim.download(), oracle.step(b, steps=3))
    sim.close()


def test_empty_instance(nbx):
    sim = nbx.Simulation(np.zeros(0, nbx.BODY_DTYPE))
    sim.step(2)
    sim.sync()
    assert len(sim.download()) == 0
    sim.close()


def test_nonfinite_reported(nbx):
    b = nbx.uniform_disc(1000)
    b["px"][10] = np.nan
    sim = nbx.Simulation(b)
    sim.step(1)
    with pytest.raises(nbx.NbxError) as e:
        sim.sync()
    assert e.value.code == 4
    sim.close()


def test_bounded_wait_expires_and_handle_recovers(nbx):
    """A device wait that nothing completes ends by its own bound (no fault,
    no hang): the host sees NBX_ERR_TIMEOUT and the handle keeps working."""
    import time
    sim = nbx.Simulation(nbx.uniform_disc(2000))
    t0 = time.perf_counter()
    sim._c(nbx.lib().nbx_debug_expire_wait(sim.h))
    with pytest.raises(nbx.NbxError) as e:
        sim.sync()
    assert e.value.code == 5  # NBX_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 60
    sim.step(3)
    sim.sync()
    assert np.isfinite(sim.download()["px"]).all()
    sim.close()


def test_capacity_errors_reported(nbx, oracle):
    b = nbx.uniform_disc(20000)
    sim = nbx.Simulation(b, node_factor=0.01)
    sim.step(1)
    with pytest.raises(nbx.NbxError) as e:
        sim.sync()
    assert e.value.code == 3
    sim.close()
    cold = nbx.cold_square(20000, 2)
    cold["px"] *= np.float32(0.3)
    cold["py"] *= np.float32(0.3)
    sim = nbx.Simulation(cold, pair_factor=0.01)
    sim.phase("iterate")  # no pending error yet
    with pytest.raises(nbx.NbxError) as e:
        sim.phase("collide")
    assert e.value.code == 3
    sim.close()


@pytest.mark.parametrize("mass,eps", [(1e30, 1.0), (2e19, 1.0), (1e6, 1e-3), (1.0, 0.0)])
def test_force_clamp_kept_where_it_can_act(nbx, oracle, mass, eps):
    """The default force pass leaves out the FLT_MAX clamp of the force law
    only where it cannot act (eps > 0 and every |m| < 1.6e19 min(1, eps^2));
    with a huge mass or tiny softening the clamp stays and the forces agree
    with the reference's clamped law."""
    b = nbx.uniform_disc(5000)
    b["mass"][0] = np.float32(mass)
    _, _, _, sb, tree = oracle.morton_build(b)
    ox, oy = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, 0.5, eps)
    sim = nbx.Simulation(b, theta=0.5, epsilon=eps)
    sim.phase("attract")
    g = sim.download()
    fin = np.isfinite(ox) & np.isfinite(oy)
    assert np.array_equal(np.isfinite(g["ax"]) & np.isfinite(g["ay"]), fin)
    e = rel_err(g["ax"][fin], g["ay"][fin], ox[fin], oy[fin])
    assert np.percentile(e, 99) < 1e-5 and e.max() < 1e-4, (np.percentile(e, 99), e.max())
    sim.close()


def _wide(nbx, scale, shift, central=None, negative=False):
    b = nbx.uniform_disc(5000)
    b["px"] *= np.float32(scale)
    b["py"] *= np.float32(scale)
    b["px"][::2] += np.float32(shift)
    b["px"][1::2] -= np.float32(shift)
    if central is not None:
        b["mass"][0] = np.float32(central)
    if negative:
        b["mass"][7] = np.float32(-3.0)
    return b


@pytest.mark.parametrize("case", ["overflowing distances", "mass-coordinate sums",
                                  "negative mass"])
def test_force_clamp_guard_wide_frame(nbx, oracle, case):
    """The clamp-free law needs every distance and centre-of-mass sum to stay
    finite: bodies beyond the upload's coordinate limit (here 1.5e19 apart,
    whose squared distances overflow, or x * m sums near 1e36) send the force
    pass back to the clamped walk, and a negative mass keeps the clamp, so
    the result is the reference's clamped law even where it gives inf: no
    NaN where the reference has a number, every infinity with its sign.
    (Where the reference gets inf - inf = NaN, the default arithmetic's
    contracted multiply-add, whose product does not round to inf first, may
    keep the inf; exact_math reproduces the NaN too.)"""
    b = {"overflowing distances": lambda: _wide(nbx, 4e14, 1.5e19),
         "mass-coordinate sums": lambda: _wide(nbx, 4e12, 2e15, central=1e18),
         "negative mass": lambda: _wide(nbx, 1.0, 0.0, negative=True)}[case]()
    _, _, _, sb, tree = oracle.morton_build(b)
    ox, oy = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, 0.5, 1.0)
    sim = nbx.Simulation(b, theta=0.5, epsilon=1.0)
    sim.phase("attract")
    g = sim.download()
    sim.close()
    for a, o in ((g["ax"], ox), (g["ay"], oy)):
        num = ~np.isnan(o)
        assert not np.isnan(a[num]).any()
        assert np.array_equal(np.isposinf(a[num]), np.isposinf(o[num]))
        assert np.array_equal(np.isneginf(a[num]), np.isneginf(o[num]))
        assert not np.isfinite(a[~num]).any()
    fin = np.isfinite(ox) & np.isfinite(oy)
    assert fin.any() or case == "overflowing distances"
    if fin.any():
        e = rel_err(g["ax"][fin], g["ay"][fin], ox[fin], oy[fin])
        assert np.percentile(e, 99) < 1e-5 and e.max() < 1e-4, (np.percentile(e, 99), e.max())
    sim = nbx.Simulation(b, theta=0.5, epsilon=1.0, exact_math=1)
    sim.phase("attract")
    g = sim.download()
    sim.close()
    assert np.array_equal(g["ax"], ox, equal_nan=True)
    assert np.array_equal(g["ay"], oy, equal_nan=True)


def test_law_error_floor(nbx):
    """The reference's fastInvSqrt law against the exact law, both summed in
    FP64 over every body: the GPU's figure against a numpy evaluation of the
    same two sums (test-side restatement)."""
    s = nbx.uniform_disc(3000)
    sim = nbx.Simulation(s)
    tg = np.arange(0, 3000, 7, dtype=np.uint32)
    got = sim.law_error(tg)
    x = s["px"].astype(np.float64)
    y = s["py"].astype(np.float64)
    m = s["mass"].astype(np.float64)
    errs = []
    for t in tg:
        dx, dy = x - x[t], y - y[t]
        d2 = dx * dx + dy * dy
        d2[t] = 1.0
        v = d2.astype(np.float32)
        g = (np.uint32(0x5f3759df) - (v.view(np.uint32) >> np.uint32(1))).view(np.float32)
        fis = (g * (np.float32(1.5) - np.float32(0.5) * v * g * g)).astype(np.float64)
        fe = m / (np.sqrt(d2) * (d2 + 1.0))
        ff = m * fis / (d2 + 1.0)
        fe[t] = ff[t] = 0.0
        ex, ey = np.sum(dx * fe), np.sum(dy * fe)
        fx, fy = np.sum(dx * ff), np.sum(dy * ff)
        errs.append(np.hypot(fx - ex, fy - ey) / np.hypot(ex, ey))
    errs = np.sort(errs)
    assert abs(got["median"] - errs[len(errs) // 2]) < 1e-6 * errs[len(errs) // 2] + 1e-9
    assert abs(got["max"] - errs[-1]) < 1e-5 * errs[-1]
    assert 1e-4 < got["median"] < 2e-3  # the bit hack's one Newton step
    sim.close()
