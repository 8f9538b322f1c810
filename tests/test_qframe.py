"""The FP32 classification of pairs from quantised positions (QFrame,
csrc/common.cuh), restated in numpy with the device's roundings, against the
reference's FP64 predicate r < h (r = sqrt of the unfused r^2, minimum image
on periodic axes; src/pre_interaction.cpp:89, include/periodic.hpp:34-59).

The classification must never contradict the predicate: "surely inside"
implies r < h and "surely outside" implies not r < h, for pairs placed at
random, within 1e-6 of h, exactly on h, across periodic faces and on the
faces of the open root box.  It must also leave only a small band to the
FP64 test."""
import numpy as np

F32 = np.float32


def _rd32(x):
    """float64 -> float32 rounded towards -inf (__double2float_rd)."""
    f = np.asarray(x, dtype=np.float64).astype(F32)
    over = f.astype(np.float64) > x
    return np.where(over, np.nextafter(f, F32(-np.inf)), f)


def _ru32(x):
    f = np.asarray(x, dtype=np.float64).astype(F32)
    under = f.astype(np.float64) < x
    return np.where(under, np.nextafter(f, F32(np.inf)), f)


def _fma32(a, b, c):
    # a*b is exact in float64 for float32 a, b; the sum rounds once to
    # float64 and once to float32 (the float64 step is far below the bound)
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def qframe(periodic, lo, rng, geo):
    if periodic:
        flo = np.array(lo, dtype=np.float64)
        s = np.array([2.0 ** 32 / L for L in rng])
    else:
        span = (geo[3] if geo[3] > 0 else 1.0) * (1.0 + 2.0 ** -8)
        flo = np.array(geo[:3]) - 0.5 * span
        s = np.full(3, 2.0 ** 31 * (1.0 - 2.0 ** -8) / span)
    inv = (1.0 / s).astype(F32)
    a = 2.0 / s.min()
    return flo, s, inv, a


def qpos(frame, periodic, x):
    flo, s, _, _ = frame
    v = (x - flo) * s
    hi = 2.0 ** 32 if periodic else 2.0 ** 31 - 64.0
    assert np.all(v >= 0) and np.all(v <= hi)
    return (np.rint(v).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32)


def qthresh(frame, h):
    a = frame[3]
    lo = (h - a) * (1.0 - 2.0 ** -20)
    hi = (h + a) * (1.0 + 2.0 ** -20)
    return np.where(lo > 0, _rd32(lo * lo), F32(0)), _ru32(hi * hi)


def qclass(frame, qi, qj):
    inv = frame[2]
    d = (qi.astype(np.int64) - qj.astype(np.int64)) & 0xFFFFFFFF
    d = np.where(d >= 2 ** 31, d - 2 ** 32, d)  # wrapping int32 difference
    near = np.all(np.abs(d) < 2 ** 30, axis=-1)
    f = d.astype(F32) * inv  # int -> float32, then one float32 product
    r2f = _fma32(f[..., 0], f[..., 0], _fma32(f[..., 1], f[..., 1], (f[..., 2] * f[..., 2]).astype(F32)))
    return near, r2f


def ref_lt(periodic, rng, xi, xj, h):
    d = xi - xj
    if periodic:
        for k in range(3):
            L = rng[k]
            c = np.stack([d[:, k], d[:, k] + L, d[:, k] - L])
            a = np.abs(c)
            pick = np.where((a[0] <= a[1]) & (a[0] <= a[2]), 0, np.where((a[1] <= a[2]) & (a[1] <= a[0]), 1, 2))
            d[:, k] = np.take_along_axis(c, pick[None], 0)[0]
    r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    return np.sqrt(r2) < h


def _pairs(rs, n, lo, hi, h, rel):
    """i uniform in the box, j at distance h (1 + rel * u) in a random direction."""
    xi = rs.uniform(lo, hi, size=(n, 3))
    u = rs.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    dist = h * (1.0 + rel * rs.uniform(-1, 1, size=(n, 1)))
    return xi, xi + u * dist


def _check(periodic, lo, hi, geo, h, xi, xj):
    rng = tuple(np.array(hi) - np.array(lo))
    if periodic:
        xj = lo + np.mod(xj - lo, rng)
    fr = qframe(periodic, lo, rng, geo)
    near, r2f = qclass(fr, qpos(fr, periodic, xi), qpos(fr, periodic, xj))
    tin, tout = qthresh(fr, h)
    truth = ref_lt(periodic, rng, xi.copy(), xj.copy(), h)
    inside = near & (r2f < tin)
    outside = near & (r2f >= tout)
    assert not np.any(inside & ~truth), "classified inside, reference says outside"
    assert not np.any(outside & truth), "classified outside, reference says inside"
    return np.mean(~inside & ~outside)


def test_open_box_random_and_near_h():
    rs = np.random.default_rng(7)
    geo = (0.01, -0.02, 0.0, 2.05)  # root centre, edge
    lo, hi = np.array(geo[:3]) - 0.85, np.array(geo[:3]) + 0.85  # j stays inside the root box
    for h in (3e-3, 0.02, 0.1):
        xi, xj = _pairs(rs, 200000, lo, hi, h, 0.5)
        band = _check(False, lo, hi, geo, h, xi, xj)
        assert band < 1e-3, band
        xi, xj = _pairs(rs, 200000, lo, hi, h, 1e-6)
        _check(False, lo, hi, geo, h, xi, xj)


def test_open_box_faces_and_exact_radius():
    rs = np.random.default_rng(11)
    geo = (0.0, 0.0, 0.0, 2.0)
    h = 0.05
    # particles on the root box's faces and corners
    xi = rs.uniform(-1, 1, size=(50000, 3))
    xi[:, rs.integers(0, 3)] = rs.choice([-1.0, 1.0], size=50000)
    u = rs.normal(size=(50000, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    xj = np.clip(xi + u * h * rs.uniform(0.5, 1.5, size=(50000, 1)), -1.0, 1.0)
    _check(False, np.full(3, -1.0), np.full(3, 1.0), geo, h, xi, xj)
    # pairs exactly h apart along an axis
    xi = rs.uniform(-0.9, 0.9, size=(50000, 3))
    xj = xi.copy()
    xj[:, 0] += h
    _check(False, np.full(3, -1.0), np.full(3, 1.0), geo, h, xi, xj)


def test_periodic_box_wraps_to_minimum_image():
    rs = np.random.default_rng(3)
    lo, hi = np.array([-0.5, 0.0, 0.0]), np.array([0.5, 0.1, 0.1])
    for h in (0.004, 0.02, 0.045):
        # near the faces, so the pairs cross them
        xi = rs.uniform(lo, hi, size=(200000, 3))
        xi[:, 1] = rs.choice([0.0, 0.1 - 1e-12, 0.05], size=200000)
        u = rs.normal(size=(200000, 3))
        u /= np.linalg.norm(u, axis=1)[:, None]
        xj = xi + u * h * (1.0 + rs.uniform(-0.3, 0.3, size=(200000, 1)))
        band = _check(True, lo, hi, None, h, xi, xj)
        # an axis difference beyond a quarter of the box goes to the FP64
        # test: with h = 0.045 in a box 0.1 wide, many do
        if h < 0.1 / 8:
            assert band < 1e-3, band
        xi, xj = _pairs(rs, 200000, lo, hi, h, 1e-7)
        _check(True, lo, hi, None, h, xi, xj)


def test_band_is_thin():
    """Away from h by more than 2e-6 relative, the classification settles
    every pair (no FP64 load)."""
    rs = np.random.default_rng(5)
    geo = (0.0, 0.0, 0.0, 2.0)
    lo, hi = np.full(3, -0.9), np.full(3, 0.9)
    h = 0.01
    xi, xj = _pairs(rs, 100000, lo, hi, h, 0.5)
    r = np.linalg.norm(xi - xj, axis=1)
    keep = np.abs(r / h - 1.0) > 2e-6
    fr = qframe(False, lo, None, geo)
    near, r2f = qclass(fr, qpos(fr, False, xi[keep]), qpos(fr, False, xj[keep]))
    tin, tout = qthresh(fr, h)
    assert np.all(near & ((r2f < tin) | (r2f >= tout)))
