"""The bench's accounting on the CPU: the endpoint-error summary the
accuracy contract is judged by, and the roofline arithmetic (achieved =
algorithmic units x flops per unit / time, frac = achieved / peak)."""
import numpy as np

import bench


def test_endpoint_errors_max_p99_and_missing_crossings():
    ref = np.zeros((5, 2))
    plane = np.zeros((5, 7))
    plane[:, 1] = [0.1e-9, -0.5e-9, 0.0, 2.0e-9, np.nan]  # x offsets
    plane[:, 2] = [0.0, 0.2e-9, -0.9e-9, 0.0, 0.0]  # y offsets
    e = bench.endpoint_errors_nm(plane, ref)
    assert e['n'] == 5
    assert e['max_nm'] == np.inf  # an electron without a crossing is infinitely wrong
    assert e['within_1nm'] == 3  # max(|dx|, |dy|) of 0.1, 0.5, 0.9 nm
    many = np.vstack([plane] + [plane[4:]] * 20)  # 21 electrons without a crossing
    e = bench.endpoint_errors_nm(many, np.zeros((len(many), 2)))
    assert e['p99_nm'] == np.inf and e['max_nm'] == np.inf and e['within_1nm'] == 3
    e = bench.endpoint_errors_nm(plane[:4], ref[:4])
    assert np.isclose(e['max_nm'], 2.0) and e['within_1nm'] == 3
    assert np.isclose(e['p99_nm'], np.percentile([0.1, 0.5, 0.9, 2.0], 99))


def test_fp64_roofline_arithmetic():
    r = bench.fp64_roofline(1e12, bench.FLOP_FIELD_PAIR, 10.0, 36.0, 'k', 'pairs')
    achieved = 1e12 * bench.FLOP_FIELD_PAIR / 10e-3 / 1e12
    assert np.isclose(r['achieved'], achieved) and np.isclose(r['frac'], achieved / 36.0)
    assert r['bound'] == 'fp64' and r['unit'] == 'TFLOP/s' and r['units'] == 1e12
    assert bench.fp64_roofline(1.0, 1, 1.0, None, 'k', 'u')['frac'] is None


def test_network_flops_per_evaluation():
    """One evaluation of the 16 -> 4 x 128 -> 32 network: 2 flops per
    multiply-add of its four matrix products."""
    assert bench.MLP_FLOP_PER_EVAL == 2 * (16 * 128 + 3 * 128 * 128 + 128 * 32) == 110592
