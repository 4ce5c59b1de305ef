"""Long-run statistics of the mixed-precision cycle against the plain FP64 device cycle on the RF-driven periodic
configuration (cfg4 physics, reduced to 64 x 64 cells, 64 particles per cell and 400 steps), over 8 seeds: the EEDF,
the electron and ion density profiles, the electron f(v_x) and the ion flux to each wall agree within their
statistical errors (Welch z-scores of the differences of the means over seeds)."""
import pytest

from edipic_b200 import PREC_FP64, PREC_MIXED
from edipic_b200.longrun import compare, run


@pytest.mark.gpu
def test_mixed_matches_fp64_statistically(tmp_path):
    kw = dict(steps=400, cells=(64, 64), ppc=64, burn_in=200, sample_every=20, workdir=str(tmp_path))
    mixed = [run(PREC_MIXED, 1000 + s, **kw) for s in range(8)]
    fp64 = [run(PREC_FP64, 1000 + s, **kw) for s in range(8)]
    z = compare(mixed, fp64)
    for k, v in z.items():
        assert v["n"] > 0, k
        assert v["max_abs_z"] < 6.0, (k, v)
        assert v["mean_z2"] < 2.0, (k, v)
    assert min(r["ion_flux"][0] + r["ion_flux"][1] for r in mixed) > 0
