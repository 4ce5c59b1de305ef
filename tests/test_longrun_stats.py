"""The statistics of the long-run comparison (edipic_b200.longrun) on synthetic per-seed samples with known answers:
the Welch scores stay small while the bias is far below the seed spread; the paired test resolves biases far below
that spread; its equivalence score is 0 for a bias inside the tolerance and large for one well outside it."""
import numpy as np

from edipic_b200.longrun import compare, compare_paired


QUANTITY_SLICES = (("eedf", 0, 40), ("ne", 40, 105), ("ni", 105, 170), ("fvx", 170, 212), ("ion_flux", 212, 214))


def _as_run(v):
    return {k: v[a:b].tolist() for k, a, b in QUANTITY_SLICES}


def _pair(bias, seed=1, seeds=8, spread=0.05, noise=1e-4):
    """Per-seed runs of the two precisions: a per-seed fluctuation of relative size `spread` shared by both runs of a
    seed (the same initial plasma), independent relative noise `noise` on each, and a relative bias `bias` of the
    first set against the second."""
    rng = np.random.default_rng(seed)
    base = 0.1 + rng.random(214)
    mixed, fp64 = [], []
    for _ in range(seeds):
        shared = base * (1.0 + spread * rng.standard_normal(base.size))
        mixed.append(_as_run(shared * (1.0 + bias) * (1.0 + noise * rng.standard_normal(base.size))))
        fp64.append(_as_run(shared * (1.0 + noise * rng.standard_normal(base.size))))
    return mixed, fp64


def test_no_bias_passes_both_analyses():
    mixed, fp64 = _pair(0.0)
    w = compare(mixed, fp64)
    p = compare_paired(mixed, fp64, rel_tol=0.01)
    for k in ("eedf", "ne", "ni", "fvx"):
        assert w[k]["max_abs_z"] < 5.0 and w[k]["mean_z2"] < 2.0, (k, w[k])
        assert p[k]["max_excess_z"] == 0.0, (k, p[k])
        # the pairing resolves relative biases far below the 5 % seed spread
        assert p[k]["detectable_bias_median"] < 1e-3, (k, p[k])


def test_small_bias_is_seen_by_the_pairing_but_inside_the_tolerance():
    mixed, fp64 = _pair(2e-3)   # 0.2 %: far below the seed spread, far above the paired resolution
    p = compare_paired(mixed, fp64, rel_tol=0.01)
    w = compare(mixed, fp64)
    for k in ("eedf", "ne", "ni", "fvx"):
        assert p[k]["max_abs_z"] > 6.0, (k, p[k])    # a plain paired bound would reject it
        assert p[k]["max_excess_z"] == 0.0, (k, p[k])  # the equivalence test at 1 % accepts it
        assert w[k]["max_abs_z"] < 5.0, (k, w[k])    # within the statistical error across seeds
        assert abs(p[k]["max_rel_bias"] - 2e-3) < 1e-3, (k, p[k])


def test_bias_beyond_the_tolerance_fails_the_equivalence_test():
    mixed, fp64 = _pair(0.03)   # 3 %: outside the 1 % tolerance
    p = compare_paired(mixed, fp64, rel_tol=0.01)
    for k in ("eedf", "ne", "ni", "fvx"):
        assert p[k]["max_excess_z"] > 6.0, (k, p[k])
