"""The float flux kernel's two ways of filling its velocity ring (tc_set_flux_staging):
16-byte cp.async chunks from every thread, and TMA tensor-map boxes on the tiles whose
halo does not wrap (the border tiles by cp.async in a second launch).  The stencils and
the arithmetic are the same, so without forcing the steps agree bit for bit; with the
constant flow rate the forcing's block sum is added in another block order."""
import numpy as np
import pytest

from cases import VV4, HW2, make_case, rel_err, within

pytestmark = pytest.mark.gpu

# NX % 64 == 0 and NY % 8 == 0 with at least 3 x 3 tiles of 64 x 8 (interior tiles exist),
# lengths the oracle transforms (2^a 3^b)
GRIDS = {"vv4_192x48": dict(scheme=VV4, NX=192, NY=48, NZ=14), "hw2_256x24": dict(scheme=HW2, NX=256, NY=24, NZ=10)}


def _run(name, staging, cfr):
    import oracle_py as op
    import turbchannel_b200 as tb

    prod, orc, zz = make_case(precision=1, **GRIDS[name])
    O = op.Oracle(orc, zz, "f64")
    O.init_channel(0, seed=12345, amp=0.1, project=True)
    v0, p0 = O.get_level(0)
    S = tb.Solver(prod, zz)
    S.set_flux_staging(staging)
    for lvl in range(4):
        S.upload_level(lvl, np.zeros_like(v0), np.zeros_like(p0))
    S.upload_level(0, v0, p0)
    if cfr:
        S.set_forcing(1, 1.0)
    cur = 0
    for it in range(4):
        S.Step(it * 1e-3, 1e-3, cur, min(it + 1, 3))
        cur = (cur + 1) % 4
    S.sync()
    out = S.download_level(cur), S.download_flux(cur)
    S.close()
    return out


@pytest.mark.parametrize("name", list(GRIDS))
def test_tma_ring_fill_matches_cp_async(name):
    (v1, p1), f1 = _run(name, 1, cfr=False)
    (v0, p0), f0 = _run(name, 0, cfr=False)
    assert np.array_equal(v1, v0) and np.array_equal(p1, p0) and np.array_equal(f1, f0)
    (v1, p1), _ = _run(name, 1, cfr=True)
    (v0, p0), _ = _run(name, 0, cfr=True)
    assert within(f"staging/{name}/cfr_vel", rel_err(v1, v0), 1e-6), rel_err(v1, v0)


def test_staging_mode_is_checked():
    import turbchannel_b200 as tb

    prod, _, zz = make_case(precision=1, **GRIDS["vv4_192x48"])
    S = tb.Solver(prod, zz)
    with pytest.raises(tb.TcError):
        S.set_flux_staging(2)
    S.close()
