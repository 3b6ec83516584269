"""Host side of the beaching hook's payload surfaces (tracking.py:236-327):
the free surface and the dry mask are formed as the reference's payload
forms them -- a LazyLerpField blends (1 - alpha) a + alpha b in the arrays'
own dtype (io.py:68-117, :499-513) -- and a 3-D dry-mask variable gives its
surface layer."""
import numpy as np
import pytest

from kelp_b200.beaching import BeachingConfig, payload_surfaces
from kelp_b200.fields import LazyLerpField, VelocityField


def _vel(eta, dry, n=6):
    return VelocityField(u=np.zeros(n), v=np.zeros(n), eta=eta, uv_layout="node", scalars={"dry": dry})


def test_surfaces_of_a_lazy_pair_blend_in_their_own_dtype():
    rng = np.random.default_rng(0)
    ea, eb = rng.normal(size=6).astype(np.float32), rng.normal(size=6).astype(np.float32)
    da, db = rng.uniform(size=(3, 6)), rng.uniform(size=(3, 6))
    vel = LazyLerpField(_vel(ea, da), _vel(eb, db), 0.3)
    eta, dry = payload_surfaces(vel, BeachingConfig(use_eta=True, dry_mask_var="dry"))
    assert eta.dtype == np.float32
    np.testing.assert_array_equal(eta, (1.0 - 0.3) * ea + 0.3 * eb)
    np.testing.assert_array_equal(dry, ((1.0 - 0.3) * da + 0.3 * db)[0])


def test_surfaces_off_missing_and_required():
    v = _vel(np.ones(6), np.zeros(6))
    assert payload_surfaces(v, BeachingConfig()) == (None, None)
    eta, dry = payload_surfaces(v, BeachingConfig(dry_mask_var="absent"))
    assert eta is None and dry is None          # the reference ignores a variable the payload lacks
    v.eta = None
    with pytest.raises(ValueError, match="eta"):
        payload_surfaces(v, BeachingConfig(use_eta=True))
