"""The byte models behind bench.py's roofline figures: the per-solve 12-word model (56 B per point-iteration in
mixed precision, 96 B in FP64, 96 B per replacement), and the bytes it counts twice when an instance's two solves
share one staging of the coefficients. No GPU."""

import bench


def _d(iters, rep=0):
    return {"numIters": iters, "replacements": rep}


def test_algorithmic_bytes_per_solve():
    n = bench.N_LLC90
    f, a = [_d(240, 9), _d(230, 9)], [_d(241, 9), _d(250, 10)]
    want = n * ((240 + 230 + 241 + 250) * 56 + (9 + 9 + 9 + 10) * 96)
    assert bench.algorithmic_bytes(f, a, "mixed") == want
    assert bench.algorithmic_bytes([_d(230)], [_d(225)], "f64") == n * (230 + 225) * 96


def test_shared_coefficients_counted_while_both_solves_iterate():
    n = bench.N_LLC90
    f, a = [_d(240), _d(230)], [_d(241), _d(250)]
    assert bench.shared_coefficient_bytes(f, a, "mixed") == n * 24 * (240 + 230)
    assert bench.shared_coefficient_bytes(f, a, "f64") == n * 48 * (240 + 230)
    # counted once, an instance-iteration with both solves moves 88 B in mixed precision (24 B of coefficients
    # and 32 B per solve), against the model's 2 x 56
    both = bench.algorithmic_bytes([_d(100)], [_d(100)], "mixed") - bench.shared_coefficient_bytes(
        [_d(100)], [_d(100)], "mixed")
    assert both == n * 100 * 88
