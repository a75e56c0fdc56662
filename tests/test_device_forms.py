"""The device code's rearrangements of the reference's arithmetic are
identities: evaluated in FP64 on seeded data, each equals the reference's
form to rounding.

* Density of a reconstructed state (lskum_device.cuh reconstruct_kstate):
  exp(t1 - log(beta)/(gamma-1)) (q_variables.F90:230-256) against
  exp(t1) (1/beta)^2 / sqrt(beta), gamma = 1.4.
* Inner iteration (primal_fp64.cu inner_sums, primal_fp32.cu): the
  reference's L sum_k w d (qt_k - qt_i), qt = q - d.dq/2
  (q_variables.F90:115-227), against dq0 + dq_i/2 - L sum_k w d (d.dq_k)/2
  with dq0 = L sum_k w d (q_k - q_i).
* FP32 flux list solve (primal_fp32.cu flux32_group): a sum(d s w) + b
  sum(d n w) against sum(d (a s w + b n w)).
"""
import numpy as np


def test_density_without_log():
    rng = np.random.default_rng(1)
    beta = rng.uniform(0.05, 5.0, 10000)
    t1 = rng.uniform(-3.0, 3.0, 10000)
    gm1 = 1.4 - 1.0
    ref = np.exp(t1 - np.log(beta) / gm1)
    temp = 0.5 / beta
    dev = np.exp(t1) * ((4.0 * temp * temp) * (1.0 / np.sqrt(beta)))
    assert np.max(np.abs(dev / ref - 1.0)) < 1e-14


def test_rearranged_inner_iteration():
    rng = np.random.default_rng(2)
    for _ in range(200):
        nb = int(rng.integers(3, 21))
        d = rng.normal(size=(nb, 2)) * rng.uniform(1e-3, 1.0)  # x_k - x_i
        w = rng.uniform(0.5, 2.0, nb)
        qi, qk = rng.normal(size=4), rng.normal(size=(nb, 4))
        dqi, dqk = rng.normal(size=(2, 4)), rng.normal(size=(nb, 2, 4))
        M = np.einsum("k,ka,kb->ab", w, d, d)
        L = np.linalg.inv(M)
        # reference: L sum w d (qt_k - qt_i)
        qti = qi[None, :] - 0.5 * (d @ dqi)                      # (nb, 4)
        qtk = qk - 0.5 * np.einsum("ka,kam->km", d, dqk)          # (nb, 4)
        ref = L @ np.einsum("k,ka,km->am", w, d, qtk - qti)
        dq0 = L @ np.einsum("k,ka,km->am", w, d, qk - qi[None, :])
        s = np.einsum("k,ka,km->am", w, d, np.einsum("ka,kam->km", d, dqk))
        dev = dq0 + 0.5 * dqi - 0.5 * (L @ s)
        assert np.max(np.abs(dev - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref)))


def test_folded_list_solve():
    rng = np.random.default_rng(3)
    for _ in range(200):
        nb = int(rng.integers(1, 9))
        dv, sw, nw = rng.normal(size=nb), rng.normal(size=nb), rng.normal(size=nb)
        a, b = rng.normal(size=2) * 10.0
        ref = a * np.sum(dv * sw) + b * np.sum(dv * nw)
        dev = np.sum(dv * (a * sw + b * nw))
        assert abs(dev - ref) <= 1e-12 * (abs(a) + abs(b)) * np.sum(np.abs(dv) * (np.abs(sw) + np.abs(nw)))
