"""Operation counts of the reference path from the instrumented oracle (the
same restatement on a counting number type): it computes what the double
oracle computes, and its per-Gauss-point counts are the figures the
kernels' rooflines quote."""
import numpy as np

from alya_sma_b200 import problem as P

NITI = P.nitinol_props(**P.NITI)


def _rotated(stretch, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] *= -1
    return q @ np.diag(stretch) @ q.T


def test_counting_instance_computes_the_oracle(oracle):
    for seed, stretch in enumerate(([1.002, 0.9994, 0.9994], [1.03, 0.991, 0.991])):
        F = _rotated(stretch, seed)
        Fc = np.ascontiguousarray(F.T).reshape(9)
        ops, s_cnt, fl_cnt = oracle.count_law160(NITI, Fc, [0.0, 0.0, 0.0])
        tau, s_ref, fl_ref = oracle.law160_kirchhoff(NITI, Fc, [0.0, 0.0, 0.0])
        assert fl_cnt == fl_ref and np.array_equal(s_cnt, s_ref)


def test_law_operation_counts(oracle):
    """compute_kirchoff_stress, averaged over rotated stretches (the
    eigensolver's QL iterations depend on the point): elastic and return-
    map points take several hundred flops each, the return map more, and
    every evaluation takes 4 logs and 1 pow (J^(-1/3))."""
    rng = np.random.default_rng(7)
    means = {}
    for kind, amp in (("elastic", 0.002), ("return map", 0.03)):
        fl_sum, n = 0.0, 0
        for seed in range(200):
            e = amp * rng.uniform(0.7, 1.0)
            F = _rotated([1 + e, 1 - 0.3 * e, 1 - 0.3 * e], 100 + seed)
            ops, _, fl = oracle.count_law160(NITI, np.ascontiguousarray(F.T).reshape(9), [0.0, 0.0, 0.0])
            assert bool(fl & 1) == (kind == "return map")
            assert ops["log"] == 4 and ops["pow"] == 1
            fl_sum += ops["add"] + ops["mul"] + ops["div"] + ops["sqrt"]
            n += 1
        means[kind] = fl_sum / n
    assert 300 <= means["elastic"] <= 900, means
    assert 400 <= means["return map"] <= 1100, means
    assert means["return map"] > means["elastic"]


def test_element_operation_counts_per_gauss_point(oracle):
    """One element of the explicit loop on the prestrained cantilever
    (geometry, F, the law, P, forces and the lumped mass the reference
    rebuilds every step): ~1.9 kflop per Gauss point."""
    prob = P.cantilever_400x40x40(nsteps=10, div=10)
    u = P.prestrain(prob, 0.01)
    tot = {}
    els = range(0, prob.nelem, 37)
    for e in els:
        ln = prob.lnods[e]
        ops, _ = oracle.count_element(prob.coord[ln].reshape(-1), u[ln].reshape(-1), prob.props[0],
                                      prob.densi[0], np.zeros(24))
        for k, v in ops.items():
            tot[k] = tot.get(k, 0) + v
    ngp = 8 * len(els)
    flops = (tot["add"] + tot["mul"] + tot["div"] + tot["sqrt"]) / ngp
    assert 1500 <= flops <= 2500, (flops, tot)
    assert tot["log"] == 4 * ngp and tot["pow"] == ngp
