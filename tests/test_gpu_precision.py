"""Covariance precision on a UTM-offset, millimetre-quantised cloud: the exact
integer sums never fail where float32 sums of world coordinates do."""
import pytest

pytestmark = pytest.mark.gpu


def test_exact_sums_survive_a_utm_offset():
    from remobench_b200 import precision
    r = precision.run(num_points=2_000_000, min_points=64)
    depths = r["per_depth"]
    assert len(depths) >= 3
    for d, res in depths.items():
        assert res["int64"]["failed_share"] == 0.0, d
        assert res["int64"]["lmin_rel_median"] < 1e-3, d
        assert res["fp32_centred"]["failed_share"] < 0.5, d
    # float32 world coordinates cannot hold 4,000 km to the millimetre
    assert max(res["fp32_naive"]["failed_share"] for res in depths.values()) > 0.5
