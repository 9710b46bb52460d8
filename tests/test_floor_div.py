"""The certificate of floor_div (csrc/common.cuh), restated in numpy float64 (IEEE round to
nearest, no contraction, as the device code with -fmad=false): the cell ids floor(x / d) of the
reference (src/common_grid.cpp:9-30, src/srd_collision.cpp:9-45) are computed as floor(q) with
q = RN(x * RN(1 / d)) whenever q lies farther than 2^-49 |q| from every integer, and by the
division otherwise. Whenever the fast path is taken it must equal floor(RN(x / d)); on exact cell
boundaries it must not be taken."""
import numpy as np

TOL = 2.0 ** -49


def floor_div(x, d):
    """(value, fast) of the device routine for arrays x and a scalar d."""
    invd = np.float64(1.0) / np.float64(d)
    q = x * invd
    f = np.floor(q)
    r = q - f
    tol = np.abs(q) * TOL
    fast = (r > tol) & (r < 1.0 - tol)
    return np.where(fast, f, np.floor(x / d)), fast


def boundary_values(d, kmax, rng, n):
    k = rng.integers(-2, kmax + 1, n).astype(np.float64)
    b = k * d
    out = [b, np.nextafter(b, -np.inf), np.nextafter(b, np.inf),
           np.nextafter(np.nextafter(b, np.inf), np.inf), np.nextafter(np.nextafter(b, -np.inf), -np.inf)]
    return np.concatenate(out)


def test_fast_path_equals_division():
    rng = np.random.default_rng(5)
    divisors = [409.6 / 2048, 0.2, 0.1, 1.0 / 3.0, 0.7, 102.4, 409.6, 819.2 / 4096, 0.3, 1.1, 2.0 ** -3]
    divisors += list(rng.uniform(0.01, 10.0, 12))
    total_fast = 0
    for d in divisors:
        d = np.float64(d)
        kmax = int(min(8192, 5000.0 / d)) + 1
        x = np.concatenate([
            boundary_values(d, kmax, rng, 20000),
            rng.uniform(-3 * d, kmax * d, 200000),
            np.array([0.0, -0.0, 5e-324, -5e-324, 1e-300, -1e-300, np.inf, -np.inf, np.nan]),
        ])
        with np.errstate(invalid="ignore", over="ignore"):
            got, fast = floor_div(x, d)
            ref = np.floor(x / d)
        ok = np.isnan(ref) & np.isnan(got) | (got == ref)
        assert ok.all(), (d, x[~ok][:5])
        total_fast += int(fast.sum())
    assert total_fast > 1_000_000  # the fast path is the common one


def test_exact_boundaries_take_the_division():
    """x = k d exactly representable with an exact quotient: q is (within rounding) the integer k,
    so the certificate must send it to the division."""
    for d in (0.25, 0.5, 2.0, 0.125):
        k = np.arange(-5, 5000, dtype=np.float64)
        x = k * d  # exact for these power-of-two divisors
        _, fast = floor_div(x, d)
        assert not fast[k != 0].any()
