"""The automatic step placement of the sweep (PipelineFunction.py:138-226)
against the oracle's restatement, on random histories with tied areas."""
import numpy as np
import pytest

from oracle import contact_oracle as oc


@pytest.mark.parametrize("seed", range(20))
def test_next_offset_matches_oracle(seed):
    from contactmechanics_b200.PipelineFunction import StepRecord, height_stats, next_offset
    rng = np.random.default_rng(seed)
    h = rng.standard_normal((12, 9))
    stats = height_stats(h)
    records = []
    for step in range(8):
        got = next_offset(records, stats)
        want = oc.auto_offset(step, [r.offset for r in records], [r.area for r in records], h)
        assert got == pytest.approx(want, rel=1e-15, abs=1e-15)
        # a fake outcome; areas drawn from a few values so that ties occur
        area = float(rng.choice([0.0, 0.05, 0.2, 0.2, 0.6, 1.0]))
        records.append(StepRecord(got, 0.0, 0.0, area, True))
