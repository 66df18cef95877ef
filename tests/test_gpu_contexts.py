"""Several engine contexts alive at once on one device.

The device-side order tables are shared by all contexts; creating a context
with another expansion order must leave the results of a live context
unchanged (the Dehnen MAC's error estimate uses C(p, k), so tables of the
wrong order would change its interaction lists)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_context_with_other_order_leaves_live_context_unchanged():
    import fmms_b200 as fx

    mass, pos = fx.gen_plummer(8192, seed=3)
    a = fx.Fmm(mass, pos, 8, 1e-6, 32)
    ra = a.run()
    b = fx.Fmm(mass, pos, 4, 1e-3, 16)
    rb = b.run()
    a.refresh(mass, pos)
    ra2 = a.run()
    assert np.array_equal(ra.accel, ra2.accel)
    assert np.array_equal(ra.pot, ra2.pot)
    assert not np.array_equal(ra.accel, rb.accel)
    c = fx.Fmm(mass, pos, 4, 1e-3, 16)
    assert np.array_equal(c.run().accel, rb.accel)


@pytest.mark.parametrize("precision", ["plain", "mixed"])
@pytest.mark.parametrize("mac", ["theta", "dehnen"])
def test_two_streams_give_the_same_bits(precision, mac):
    """An evaluation on two streams (walk and lists beside the upward pass,
    P2P beside M2L) gives the bits of the same evaluation on one stream."""
    import fmms_b200 as fx

    mass, pos = fx.gen_plummer(16384, seed=11)
    kw = dict(mac=mac, theta=0.5, softening=1e-3, precision=precision)
    out = []
    for overlap in (False, True):
        r = fx.Fmm(mass, pos, 8, 1e-6, 32, overlap=overlap, **kw).run()
        out.append((r.accel, r.pot))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
