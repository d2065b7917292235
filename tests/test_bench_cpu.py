"""bench.py's CPU-baseline arithmetic: iterations to the tolerance from the
relative residuals of the timed outer iterations (one or several), the
number the reference arm's solves/s rests on."""
import importlib.util
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location("fg_bench", os.path.join(HERE, "..", "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_one_timed_iteration_uses_its_own_factor():
    rho, n = bench.extrapolate_iterations(1.0, [0.1])
    assert math.isclose(rho, 0.1)
    assert math.isclose(n, math.log(bench.RTOL) / math.log(0.1))


def test_several_iterations_use_the_factor_after_the_first():
    res = [0.05, 0.005, 0.0005]
    rho, n = bench.extrapolate_iterations(1.0, res)
    assert math.isclose(rho, 0.1)
    assert math.isclose(n, 1 + math.log(bench.RTOL / 0.05) / math.log(0.1))


def test_no_reduction_gives_no_number():
    rho, n = bench.extrapolate_iterations(1.0, [1.2])
    assert n != n  # nan: the arm then reports 0 solves/s rather than a made-up rate
