"""Settings the reference refuses are refused here with a status, before any work: Ewald with ceil(hCut) > 3
(ryoanji/src/ryoanji/nbody/ewald.hpp:52-60 asserts it; the k-space tables here are sized for it), negative settings
and a zero alpha with Ewald on. Open boxes ignore the Ewald settings, as the reference's open solves do."""
import numpy as np
import pytest
import torch

from ryoanji_b200 import datasets as ds

pytestmark = pytest.mark.gpu


def _arrays(p):
    dev = [torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]
    return dev + [torch.empty(p.n, device="cuda") for _ in range(4)]


@pytest.mark.parametrize("settings", [dict(hCut=3.5), dict(hCut=-1.0), dict(lCut=-0.5), dict(alpha_scale=0.0)])
def test_solve_refuses_ewald_settings_the_reference_refuses(settings):
    import ryoanji_b200 as ryo
    p = ds.periodic_box(2000, seed=9, eps=0.01)
    box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    params = ryo.SolveParams(box=box, ewald=ryo.EwaldSettings(**settings))
    with pytest.raises(ryo.RyoError) as e:
        ryo.solve(*_arrays(p), params=params)
    assert e.value.status == ryo._abi.ERR_BAD_ARG and "ewald" in str(e.value)
    # the same settings are not used, hence not checked, for an open box
    params = ryo.SolveParams(ewald=ryo.EwaldSettings(**settings))
    ryo.solve(*_arrays(ds.uniform_cube(2000, seed=10, eps=0.01)), params=params)


def test_ewald_at_the_limit_still_runs():
    """hCut = 3 (ceil 3) is the largest the reference accepts"""
    import ryoanji_b200 as ryo
    p = ds.periodic_box(2000, seed=11, eps=0.01)
    box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    arrays = _arrays(p)
    ryo.solve(*arrays, params=ryo.SolveParams(box=box, ewald=ryo.EwaldSettings(hCut=3.0)))
    assert all(bool(torch.isfinite(a).all()) for a in arrays[5:])


def test_engine_and_particle_ewald_refuse_them_too():
    import ryoanji_b200 as ryo
    bad = ryo.EwaldSettings(hCut=3.5)
    with pytest.raises(ryo.RyoError) as e:
        ryo.Engine(ryo.SolveParams(ewald=bad))
    assert e.value.status == ryo._abi.ERR_BAD_ARG
    p = ds.periodic_box(500, seed=12, eps=0.01)
    dev = [torch.from_numpy(a).cuda() for a in (p.x, p.y, p.z, p.m, p.h)]
    targets = torch.arange(0, 500, 50, dtype=torch.int64, device="cuda")
    with pytest.raises(ryo.RyoError) as e:
        ryo.ewald_targets_f64(targets, *dev, L=1.0, ewald=bad)
    assert e.value.status == ryo._abi.ERR_BAD_ARG
    np.testing.assert_equal(p.n, 500)
