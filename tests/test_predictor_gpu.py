"""Device-resident Hermite state and predictor vs the FP64 oracle
(xbpredall.F:49-61).  The predictor is FP64 on the GPU: agreement to a few
ulp (relative 1e-14), and nb6_predict_send_ produces the same regular-force
results as a host prediction followed by gpunb_send_."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


def _state(n, seed):
    from nb6b200 import ics
    rng = np.random.default_rng(seed)
    cl = ics.plummer(n, seed=seed, imf=True)
    return {"body": cl.mass, "t0": -rng.integers(0, 32, n) / 4096.0, "x0": cl.pos,
            "x0dot": cl.vel, "f": rng.normal(size=(n, 3)) * 0.3,
            "fdot": rng.normal(size=(n, 3)) * 0.1, "rs": cl.rs, "dtr": cl.dtr}


def _set(raw, s):
    n = len(s["body"])
    a = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in s.items()}
    raw.nb6_state_open_(C.byref(C.c_int(n)))
    raw.nb6_state_set_(C.byref(C.c_int(n)), a["body"].ctypes.data_as(dp),
                       a["t0"].ctypes.data_as(dp), a["x0"].ctypes.data_as(dp),
                       a["x0dot"].ctypes.data_as(dp), a["f"].ctypes.data_as(dp),
                       a["fdot"].ctypes.data_as(dp))
    return a


@pytest.mark.parametrize("n", [1, 257, 100000])
def test_predict_matches_oracle(nb6, orc, n):
    raw = nb6.lib
    s = _set(raw, _state(n, n))
    try:
        x = np.zeros((n, 3))
        xd = np.zeros((n, 3))
        t = C.c_double(1.0 / 256)
        raw.nb6_predict_(C.byref(t), x.ctypes.data_as(dp), xd.ctypes.data_as(dp))
        ox, oxd = orc.predict(t.value, s["t0"], s["x0"], s["x0dot"], s["f"], s["fdot"])
        np.testing.assert_allclose(x, ox, rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(xd, oxd, rtol=1e-14, atol=1e-15)
    finally:
        raw.nb6_state_close_()


def test_state_update_scatter(nb6, orc):
    raw = nb6.lib
    n = 5000
    s = _set(raw, _state(n, 2))
    try:
        rng = np.random.default_rng(3)
        idx = np.sort(rng.choice(n, 400, replace=False)).astype(np.int32)
        for k in ("x0", "x0dot", "f", "fdot"):
            s[k][idx] += rng.normal(size=(len(idx), 3)) * 1e-3
        s["t0"][idx] = 1.0 / 1024
        sub = {k: np.ascontiguousarray(s[k][idx]) for k in ("body", "t0", "x0", "x0dot", "f", "fdot")}
        one = (idx + 1).astype(np.int32)
        raw.nb6_state_update_(C.byref(C.c_int(len(idx))), one.ctypes.data_as(ip),
                              sub["body"].ctypes.data_as(dp), sub["t0"].ctypes.data_as(dp),
                              sub["x0"].ctypes.data_as(dp), sub["x0dot"].ctypes.data_as(dp),
                              sub["f"].ctypes.data_as(dp), sub["fdot"].ctypes.data_as(dp))
        x = np.zeros((n, 3))
        xd = np.zeros((n, 3))
        t = C.c_double(1.0 / 512)
        raw.nb6_predict_(C.byref(t), x.ctypes.data_as(dp), xd.ctypes.data_as(dp))
        ox, oxd = orc.predict(t.value, s["t0"], s["x0"], s["x0dot"], s["f"], s["fdot"])
        np.testing.assert_allclose(x, ox, rtol=1e-14, atol=1e-15)
    finally:
        raw.nb6_state_close_()


def test_predict_send_equals_host_predict_then_send(nb6, orc):
    raw = nb6.lib
    n = 6000
    s = _set(raw, _state(n, 5))
    t = C.c_double(3.0 / 1024)
    ox, oxd = orc.predict(t.value, s["t0"], s["x0"], s["x0dot"], s["f"], s["fdot"])
    ifirst, nn = 101, n - 100          # as GPUNB_SEND(NN, BODY(IFIRST), ...)
    isel = np.arange(0, nn, 5)
    h2 = s["rs"][100:][isel] ** 2
    dtr = s["dtr"][100:][isel]
    try:
        nb6.gpunb_open(n + 10, 0)
        raw.nb6_predict_send_(C.byref(t), C.byref(C.c_int(ifirst)), C.byref(C.c_int(nn)))
        a1, j1, p1, l1 = nb6.gpunb_regf(h2, dtr, ox[100:][isel], oxd[100:][isel], 512, 400, 0)
        nb6.gpunb_send(s["body"][100:], ox[100:], oxd[100:])
        a2, j2, p2, l2 = nb6.gpunb_regf(h2, dtr, ox[100:][isel], oxd[100:][isel], 512, 400, 0)
        nb6.gpunb_close()
        np.testing.assert_array_equal(l1, l2)
        np.testing.assert_allclose(a1, a2, rtol=1e-12)
        np.testing.assert_allclose(p1, p2, rtol=1e-12)
    finally:
        raw.nb6_state_close_()
