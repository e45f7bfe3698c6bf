"""The device block clock (nb6_blocks_run_) and the device correctors'
state calls, at the C ABI: the block it picks is the host's choice (the
bodies with the smallest T0 + STEP), its corrector rows equal
nb6_irr_correct_'s for that set bit for bit, the due list is the rows'
regular-due flags in ascending order, and the stop reasons follow
tlimit and max_blocks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(seed, n=3000, lmax=128):
    """A Plummer cluster at t0 = 0 with random power-of-two steps, lists
    from the FP64 oracle's regular call, forces from a random draw."""
    from nb6b200 import ics
    cl = ics.plummer(n, seed=seed, imf=True)
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(n, 3)) * 0.05
    fd = rng.normal(size=(n, 3)) * 0.01
    step = 2.0 ** -rng.integers(6, 10, n).astype(float)
    stepr = np.maximum(step, 2.0 ** -rng.integers(4, 7, n).astype(float))
    stepr[::3] = step[::3]         # a third of the bodies due a regular step with their first
    t0 = np.zeros(n)
    d = np.linalg.norm(cl.pos[:, None, :] - cl.pos[None, :200, :], axis=2)
    lists = np.zeros((n, lmax), dtype=np.int32)
    for i in range(n):
        nb = np.nonzero((d[i] < 0.3) & (np.arange(200) != i))[0][: lmax - 9] + 1
        lists[i, 0] = len(nb)
        lists[i, 1:1 + len(nb)] = nb
    fi = rng.normal(size=(n, 3)) * 0.1
    fid = rng.normal(size=(n, 3)) * 0.01
    fr = rng.normal(size=(n, 3)) * 0.1
    frd = rng.normal(size=(n, 3)) * 0.01
    return dict(cl=cl, f=f, fd=fd, t0=t0, step=step, stepr=stepr, lists=lists, fi=fi, fid=fid, fr=fr, frd=frd,
                lmax=lmax)


def _open(nb6, S):
    cl = S["cl"]
    n = cl.n
    nb6.irr_open(n, S["lmax"], 0)
    nb6.irr_set_jp_all(cl.pos, cl.vel, S["f"], S["fd"], cl.mass, S["t0"])
    for a in range(1, n + 1):
        nb6.irr_set_list(a, S["lists"][a - 1])
    nb6.hermite_open(0.02, 0.125, 2.0 ** -24)
    nb6.hermite_set_all(S["fi"], S["fid"], S["fr"], S["frd"], S["step"], np.zeros(n), S["stepr"], cl.rs)


@pytest.mark.parametrize("due_sort_min", [None, "0"])
def test_block_clock_first_block_equals_host_choice_and_corrector(nb6, monkeypatch, due_sort_min):
    """due_sort_min "0": the due list through the radix sort instead of the
    one-launch ranking."""
    if due_sort_min is not None:
        monkeypatch.setenv("NB6_DUE_SORT_MIN", due_sort_min)
    S = _state(5)
    n = S["cl"].n
    tmin = (S["t0"] + S["step"]).min()
    act_host = np.nonzero(S["t0"] + S["step"] == tmin)[0] + 1
    _open(nb6, S)
    try:
        r0 = nb6.blocks_run(tmin / 2, 10)                 # the first block is past the limit
        assert r0["reason"] == 2 and r0["blocks"] == 0
        r1 = nb6.blocks_run(1.0, 1)                       # one block
        assert r1["blocks"] == 1 and r1["tblock"] == tmin and r1["nact"] == len(act_host)
        assert r1["reason"] in (0, 1)
        addr, rows = nb6.blocks_active(n)
        due, xv = nb6.blocks_regular(n)
        state = nb6.hermite_get(1, n)
    finally:
        nb6.irr_close(0)
    order = np.argsort(addr)
    np.testing.assert_array_equal(addr[order], act_host)
    rows = rows[order]
    # the due list: the rows' regular-due flags, ascending, with x0 and v0
    flagged = act_host[rows[:, 19] != 0]
    np.testing.assert_array_equal(due, flagged)
    np.testing.assert_array_equal(xv, rows[rows[:, 19] != 0][:, :6])
    assert r1["reason"] == 1 and len(flagged) > 0
    # the same set through nb6_irr_correct_ on a fresh copy of the state
    _open(nb6, S)
    try:
        ref = nb6.irr_correct(tmin, act_host)
    finally:
        nb6.irr_close(0)
    np.testing.assert_array_equal(rows, ref)
    # the resident state took the corrected values
    np.testing.assert_array_equal(state[act_host - 1][:, :6], ref[:, :6])
    np.testing.assert_array_equal(state[act_host - 1][:, 24], np.full(len(act_host), tmin))


def test_block_clock_runs_to_the_limit(nb6):
    """Blocks run back to back until a regular step is due or the limit is
    passed; every block time is a multiple of the smallest step, increasing."""
    S = _state(6)
    S["stepr"][:] = 1.0            # no regular step due before t = 1
    n = S["cl"].n
    _open(nb6, S)
    try:
        r = nb6.blocks_run(0.25, 100000)
        state = nb6.hermite_get(1, n)
    finally:
        nb6.irr_close(0)
    assert r["reason"] == 2 and r["blocks"] > 1 and r["tblock"] <= 0.25
    t0 = state[:, 24]
    step = state[:, 25]
    assert np.all(t0 <= 0.25) and np.all(t0 + step > 0.25 - 1e-15)
    assert r["irr_steps"] >= n


@pytest.mark.parametrize("stepr_all", [None, 1.0])
def test_persistent_and_graph_forms_agree_bit_for_bit(nb6, stepr_all):
    """The persistent form (one cooperative launch per call, grid barriers
    between the phases of a block) and the graph form (two launches per
    block) give the same blocks, active sets, corrector rows, due lists and
    final state.  stepr_all = 1.0: no regular step due, the run ends at the
    time limit after many blocks; None: it stops at the first block with a
    regular-due body."""
    S = _state(7)
    if stepr_all is not None:
        S["stepr"][:] = stepr_all
    n = S["cl"].n
    out = {}
    for persistent in (True, False):
        _open(nb6, S)
        try:
            nb6.blocks_mode(persistent)
            runs = [nb6.blocks_run(0.25, 100000) for _ in range(3 if stepr_all is None else 1)]
            addr, rows = nb6.blocks_active(n)
            due, xv = nb6.blocks_regular(n)
            out[persistent] = (runs, addr, rows, due, xv, nb6.hermite_get(1, n))
        finally:
            nb6.blocks_mode(False)
            nb6.irr_close(0)
    (r1, a1, w1, d1, x1, s1), (r0, a0, w0, d0, x0, s0) = out[True], out[False]
    assert r1 == r0
    assert sum(r["blocks"] for r in r1) > (1 if stepr_all is None else 10)
    o1, o0 = np.argsort(a1), np.argsort(a0)
    np.testing.assert_array_equal(a1[o1], a0[o0])
    np.testing.assert_array_equal(w1[o1], w0[o0])
    np.testing.assert_array_equal(d1, d0)
    np.testing.assert_array_equal(x1, x0)
    np.testing.assert_array_equal(s1, s0)


def test_persistent_form_in_the_ensemble_driver_bit_for_bit(nb6):
    """The ensemble driver with the device block clock, run once per form
    (the library call switches the form the driver's calls use): same
    blocks, steps, state and energies."""
    from nb6b200 import drive, ics
    ours = drive.backend_paths("nb6b200")
    cls = [ics.plummer(n, seed=40 + n, imf=True) for n in (700, 1500, 2300)]
    kw = dict(batched=True, tcrit=0.25, dt_out=0.125, dev_corrector=3)
    runs = {}
    for persistent in (True, False):
        nb6.blocks_mode(persistent)
        try:
            runs[persistent] = drive.run_ensemble(ours, cls, **kw)
        finally:
            nb6.blocks_mode(False)
    a, b = runs[True], runs[False]
    for key in ("blocks", "irr_steps", "reg_steps", "reg_calls", "nb_sum"):
        assert a.stats[key] == b.stats[key], key
    assert a.stats["blocks"] > 100
    for c in range(len(cls)):
        np.testing.assert_array_equal(a.x[c], b.x[c])
        np.testing.assert_array_equal(a.v[c], b.v[c])
    np.testing.assert_array_equal(a.energy, b.energy)


def _ks_table(S, seed, npair=25):
    """Perturbed pairs among the bodies the neighbour lists hold (the first
    200), components about each c.m. body's position, random perturbers."""
    cl = S["cl"]
    n = cl.n
    rng = np.random.default_rng(seed)
    cm = np.sort(rng.choice(200, npair, replace=False)) + 1
    m = cl.mass[cm - 1]
    q = rng.uniform(0.2, 0.8, npair)
    d = rng.normal(size=(npair, 3))
    d *= (2e-3 / np.linalg.norm(d, axis=1))[:, None]
    dv = rng.normal(size=(npair, 3)) * 0.3
    x, v = cl.pos[cm - 1], cl.vel[cm - 1]
    xk = np.stack([x + (1 - q)[:, None] * d, x - q[:, None] * d], axis=1)
    vk = np.stack([v + (1 - q)[:, None] * dv, v - q[:, None] * dv], axis=1)
    mk = np.stack([q * m, (1 - q) * m], axis=1)
    pofs, plist = [0], []
    for p in range(npair):
        k = int(rng.integers(0, 20))
        others = np.delete(np.arange(1, n + 1), cm[p] - 1)
        plist.extend(rng.choice(others, k, replace=False).tolist())
        pofs.append(len(plist))
    return cm, xk, vk, mk, np.array(pofs, dtype=np.int32), np.array(plist, dtype=np.int32)


def test_block_clock_with_ks_pairs_equals_corrector_call(nb6):
    """With a KS pair table set, a block of the device clock (the corrected
    neighbour walk inside blk_step) gives nb6_irr_correct_'s rows for the
    same active set, bit for bit."""
    S = _state(9)
    n = S["cl"].n
    table = _ks_table(S, 9)
    tmin = (S["t0"] + S["step"]).min()
    act_host = np.nonzero(S["t0"] + S["step"] == tmin)[0] + 1
    assert np.intersect1d(act_host, table[0]).size > 0 or len(act_host) > 20
    _open(nb6, S)
    try:
        nb6.ks_set(*table)
        r1 = nb6.blocks_run(1.0, 1)
        addr, rows = nb6.blocks_active(n)
    finally:
        nb6.irr_close(0)
    assert r1["blocks"] == 1 and r1["nact"] == len(act_host)
    _open(nb6, S)
    try:
        nb6.ks_set(*table)
        ref = nb6.irr_correct(tmin, act_host)
        nb6.ks_set([], [], [], [], [0], [])
        plain = nb6.irr_correct(tmin, act_host)
    finally:
        nb6.irr_close(0)
    order = np.argsort(addr)
    np.testing.assert_array_equal(addr[order], act_host)
    np.testing.assert_array_equal(rows[order], ref)
    assert np.any(ref[:, 6:9] != plain[:, 6:9])          # the pairs changed some forces


def test_block_clock_forms_agree_with_ks_pairs(nb6):
    """The persistent and graph forms with a KS pair table set (their
    corrected walks) over a run of many blocks: same final state."""
    S = _state(10)
    S["stepr"][:] = 1.0
    n = S["cl"].n
    table = _ks_table(S, 10)
    out = {}
    for persistent in (True, False):
        _open(nb6, S)
        try:
            nb6.ks_set(*table)
            nb6.blocks_mode(persistent)
            out[persistent] = (nb6.blocks_run(0.125, 100000), nb6.hermite_get(1, n))
        finally:
            nb6.blocks_mode(False)
            nb6.irr_close(0)
    assert out[True][0] == out[False][0] and out[True][0]["blocks"] > 10
    np.testing.assert_array_equal(out[True][1], out[False][1])
