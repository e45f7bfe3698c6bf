"""Initial-condition formats of the reference (data.F) and the Henon
rescaling (scale.F)."""
import numpy as np


def test_nbody_format_round_trip_and_fortran_exponents(tmp_path):
    from nb6b200 import ics, io
    cl = ics.plummer(300, seed=5, imf=True)
    p = tmp_path / "dat.10"
    io.write_nbody(p, cl.mass, cl.pos, cl.vel)
    m, x, v = io.read_nbody(p)
    np.testing.assert_array_equal(m, cl.mass)
    np.testing.assert_array_equal(x, cl.pos)
    np.testing.assert_array_equal(v, cl.vel)
    # list-directed records: commas, D exponents, several records per line
    q = tmp_path / "dat.10b"
    q.write_text("1.0D-03, 0.5 0.25 -1.5D+00 0.1 0.2 0.3\n2.0d-03 1 2 3\n 4 5 6\n")
    m, x, v = io.read_nbody(q)
    np.testing.assert_allclose(m, [1e-3, 2e-3])
    np.testing.assert_allclose(x[0], [0.5, 0.25, -1.5])
    np.testing.assert_allclose(v[1], [4, 5, 6])
    m, _, _ = io.read_nbody(p, n=10)
    assert m.shape == (10,)


def test_tree_format(tmp_path):
    from nb6b200 import io
    rng = np.random.default_rng(1)
    m, x, v = rng.random(5), rng.normal(size=(5, 3)), rng.normal(size=(5, 3))
    p = tmp_path / "tree.dat"
    with open(p, "w") as f:
        f.write("5\n3\n0.0\n")
        for a in m:
            f.write(f"{float(a)!r}\n")
        for r in x:
            f.write(" ".join(repr(float(c)) for c in r) + "\n")
        for r in v:
            f.write(" ".join(repr(float(c)) for c in r) + "\n")
    m2, x2, v2 = io.read_tree(p)
    np.testing.assert_array_equal(m2, m)
    np.testing.assert_array_equal(x2, x)
    np.testing.assert_array_equal(v2, v)


def test_to_henon_units():
    from nb6b200 import io
    rng = np.random.default_rng(2)
    m = rng.random(400) + 0.5
    x = rng.normal(size=(400, 3)) * 3.0 + 7.0
    v = rng.normal(size=(400, 3)) * 0.2
    mh, xh, vh = io.to_henon(m, x, v, q_vir=0.5)
    w = io.potential_energy(mh, xh)
    k = 0.5 * float((mh * (vh * vh).sum(1)).sum())
    assert abs(mh.sum() - 1) < 1e-14
    assert abs(k + w + 0.25) < 1e-12
    assert abs(k / abs(w) - 0.5) < 1e-12
    assert np.abs((mh[:, None] * xh).sum(0)).max() < 1e-12
