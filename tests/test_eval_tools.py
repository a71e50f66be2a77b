"""Host logic of the measurement drivers (no GPU): the equal-error time of
the guided comparison and the uneven job mix of the batch comparison."""
import math

import numpy as np

from azimuth_b200.batch_eval import job_specs
from azimuth_b200.guiding_eval import _relmse, _time_to


def test_time_to_interpolates_in_log_error():
    curve = [(1.0, 1e-2), (2.0, 1e-3), (3.0, 1e-4)]
    # halfway between 1e-2 and 1e-3 in log error is reached halfway between 1 s and 2 s
    assert math.isclose(_time_to(curve, math.sqrt(1e-2 * 1e-3)), 1.5, rel_tol=1e-12)
    assert _time_to(curve, 1e-3) == 2.0
    assert _time_to(curve, 1e-5) is None          # never reached
    assert _time_to(curve, 1.0) == 1.0            # reached by the first point
    # an error curve that rises before it falls is not interpolated backwards
    assert _time_to([(1.0, 1e-3), (2.0, 2e-3), (3.0, 5e-4)], 1e-3) == 1.0


def test_relmse_is_zero_for_the_reference_and_scale_free_above_the_floor():
    rng = np.random.default_rng(0)
    ref = rng.uniform(10.0, 20.0, (4, 5, 3))
    assert _relmse(ref, ref) == 0.0
    a = _relmse(ref * 1.01, ref)
    b = _relmse(ref * 101.0, ref * 100.0)   # same relative error, far above the 1e-2 floor
    assert math.isclose(a, b, rel_tol=1e-3)


def test_job_mix_is_seeded_and_within_its_ranges():
    a, b = job_specs(256, 0), job_specs(256, 0)
    assert a == b and job_specs(256, 1) != a
    for j, s in enumerate(a):
        assert s["config"] in (0, 1, 2)
        assert 5 <= s["max_depth"] <= 16 and 1 <= s["spp"] <= 256
        assert 8 <= s["width"] and 8 <= s["height"]
        assert 64 * 64 / 2 <= s["width"] * s["height"] <= 1024 * 1024 * 16 / 9 * 1.1
        assert s["guided"] == (j % 2 == 1)
