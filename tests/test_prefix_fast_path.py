"""The statistics fast path's claims (tm_prefix.cuh, prefix_stats_fast), checked on the CPU.

For a window in one prefix block, the full derivation (prefix_sums_one_block followed by
prefix_stats_tail) bounds the variance error by e_var, the std's relative error by rel_sd
and the mean's error by e_mu. The fast path replaces the per-window terms by constants of
the block (a, b from the block total of squares T2) and claims, whenever
(a + 2 |mu_c| b) / m <= 0.9e-7 var and mu_c^2 <= 1e6 var:
  * the full e_var <= 1e-4 var (the statistics are trusted),
  * the full rel_sd <= kFastRelSd = 6.6e-7,
  * the full e_mu <= b / m + 1.3e-7 |mu| + 1.9e-7 |c|.
Here both sides are evaluated in float32 in the device code's order, over seeded windows
of prefix blocks with offsets, loud and quiet stretches and means far from the block
centre, and the claims are checked wherever the fast condition holds.
"""
import numpy as np

F = np.float32
GAMMA = 80.0 * 1.1102230246251565e-16
EPS64 = 1.1102230246251565e-16
FAST_REL_SD = F(6.6e-7)


def _sqrt_up(x):
    x = F(x)
    return F(x * F(1.0 / np.sqrt(np.float64(x))) * F(1.0 + 1.9073486e-06)) if x > 0 else F(0.0)


def _block(rng, n=1 << 16):
    x = rng.normal(size=n) * rng.uniform(0.01, 10.0) + rng.uniform(-1e3, 1e3)
    a = int(rng.integers(0, n - 4000))
    x[a:a + int(rng.integers(10, 4000))] *= rng.choice([1e-3, 1e3])
    x[int(rng.integers(0, n - 2000)):][:2000] += rng.uniform(-50, 50)
    x = x.astype(np.float32).astype(np.float64)
    c = float(np.mean(x))
    d = x - c
    Q = np.zeros((n + 1, 2))
    Q[1:, 0] = np.cumsum(d)
    Q[1:, 1] = np.cumsum(d * d)
    return Q, c


def _full(Qa, Qb, na, nb, m, inv_m, c):
    fg, fe = F(GAMMA) * F(1.01), F(EPS64) * F(1.01)
    qa, qb = F(Qa[1]), F(Qb[1])
    s1, s2 = Qb[0] - Qa[0], Qb[1] - Qa[1]
    e_s2 = fg * (qa + qb)
    e_s1 = F(1.001) * fg * _sqrt_up(F(2.0) * (F(na) * qa + F(nb) * qb))
    mu_c = s1 * inv_m
    var = -mu_c * mu_c + s2 * inv_m
    fvar, fmu = F(var), F(mu_c)
    fm, fim = F(m), F(inv_m) * F(1.0 + 1.1920929e-07)
    fs2 = fm * (fvar + fmu * fmu) * F(1.0001)
    e_s2 = e_s2 + F(4.0) * fe * fs2
    e_s1 = e_s1 + F(4.0) * fe * fm * abs(fmu)
    e_var = (e_s2 + F(2.0) * abs(fmu) * e_s1 + F(8.0) * fe * fs2) * fim * F(1.0001)
    cf = F(c)
    iv = F(1.0 / np.sqrt(np.float64(fvar))) if fvar > 0 else F(np.inf)
    mu = fmu + cf
    rel_sd = F(0.5) * e_var * iv * iv * F(1.001) + F(6.0e-7)
    e_mu = e_s1 * fim + F(1.2e-7) * (abs(mu) + abs(cf)) + F(4.0) * fe * abs(mu) + F(6.0e-8) * abs(cf)
    return var, fvar, fmu, e_var, rel_sd, e_mu, mu, cf, fim


def test_fast_path_claims_hold():
    rng = np.random.default_rng(77)
    fg = F(GAMMA) * F(1.01)
    checked, rejected = 0, 0
    for _ in range(6):
        Q, c = _block(rng)
        n = len(Q) - 1
        T2 = F(Q[n, 1]) * F(1.00001)
        a = F(2.0) * fg * T2 * F(1.00001)
        b = F(1.001) * fg * F(512.0) * _sqrt_up(T2) * F(1.00001)
        for _ in range(3000):
            m = int(rng.choice([16, 100, 1024, 4096, 16384]))
            j = int(rng.integers(0, n - m))
            inv_m = 1.0 / m
            var, fvar, fmu, e_var, rel_sd, e_mu, mu, cf, fim = _full(Q[j], Q[j + m], j, j + m, m, inv_m, c)
            fast = (fvar > F(2e-22) and fvar < F(1e36) and fmu * fmu <= F(1e6) * fvar and
                    (a + F(2.0) * abs(fmu) * b) * fim <= F(0.9e-7) * fvar)
            if not fast:
                rejected += 1
                continue
            checked += 1
            assert e_var <= F(1e-4) * fvar
            assert rel_sd <= FAST_REL_SD, (rel_sd, m)
            assert e_mu <= b * fim + F(1.3e-7) * abs(mu) + F(1.9e-7) * abs(cf)
    assert checked > 10000, checked
    assert rejected > 0  # quiet windows in loud blocks, and means far from the centre, take the full bound
