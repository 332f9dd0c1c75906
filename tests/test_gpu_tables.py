"""Tables of a context: the identity-emit table and its finiteness check.

fx_set_tables builds, on the device, the emitted value of every raw sample
(the output of every unattempted channel).  A LUT holding a non-finite value
is refused there with the reference's "work RGB must be finite" error
instead of failing later inside a frame.
"""

from __future__ import annotations

import numpy as np
import pytest

from fauxice_b200 import _lib
from fauxice_b200.engine import factor_tables, response_lut

pytestmark = pytest.mark.gpu


def test_non_finite_lut_is_refused_and_the_context_stays_usable():
    lut = response_lut().copy()
    high, low = factor_tables()
    ctx = _lib.Context(0)
    try:
        bad = lut.copy()
        bad[12345] = np.nan
        with pytest.raises(_lib.LibraryError) as raised:
            ctx.set_tables(bad, high, low)
        assert raised.value.status == 6  # FX_ERR_NONFINITE_WORK
        assert "finite" in str(raised.value)
        ctx.set_tables(lut, high, low)  # the pinned tables are accepted again
    finally:
        ctx.close()
