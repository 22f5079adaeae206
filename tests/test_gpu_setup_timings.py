"""amg_setup_timings: the set-up's device time by phase (CUDA events at the phase
boundaries).  On a 64x64, 3-level mixed-precision context with test-vector smoothing and one
bootstrap pass every phase is non-negative, the smoothing, orthonormalisation, coarse-link,
bootstrap and mixed-copy phases are positive, and the phases add up to the set-up's own
device time (amg_last_timings) within 10 %."""
import pytest

pytestmark = pytest.mark.gpu


def test_setup_phases_add_up_to_the_setup():
    from amg_schwingermodel_b200 import AMGContext
    from amg_schwingermodel_b200.inputs import gauge_field
    with AMGContext(64, 64, [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]], -0.1, precision=1, nit=1) as ctx:
        ctx.set_gauge(gauge_field(64, 64, 3.0, 11))
        ctx.setup()
        ph = ctx.setup_timings()
        setup_ms, _ = ctx.timings()
    print(ph, setup_ms)
    assert all(v >= 0 for v in ph.values()), ph
    for k in ("smoothing", "orthonormalisation", "coarse_links", "bootstrap", "mixed_copies"):
        assert ph[k] > 0, (k, ph)
    assert abs(sum(ph.values()) - setup_ms) <= 0.1 * setup_ms, (ph, setup_ms)
