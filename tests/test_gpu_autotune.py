"""The autotuner on the GPU: every candidate launch shape runs, the tuned step still matches
the FP64 oracle (1e-5 normwise, the FP32 bar), the cache written for this GPU restores the
same choices on a new context, and an invalid choice is rejected."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import autotune
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

GAMMA = 9.784756683727565


@pytest.mark.parametrize("order", [osc.ORDER_ANY, osc.ORDER_CELL_SORTED])
def test_tune_then_apply(oracle, tmp_path, order):
    torch = pytest.importorskip("torch")
    n = (32, 32, 64)
    x, y, z = gendist(300_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=61)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umin + (np.array(n) - 1) * delta, delta=delta, gamma=GAMMA)
    if order != osc.ORDER_ANY:
        p = np.argsort(osc.cell_keys(mesh, x, y, z), kind="stable")
        x, y, z = (np.ascontiguousarray(a[p]) for a in (x, y, z))
    tx, ty, tz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    E = torch.empty((len(x), 3), dtype=torch.float64, device="cuda")
    cache = str(tmp_path / "autotune.json")
    with osc.Context(0) as c:
        def step():
            osc.space_charge_step_dev(c, mesh, tx, ty, tz, E, total_charge=1e-9, resize_mesh=False,
                                      precision=osc.PREC_FP32)
        res = autotune.tune(c, step, n, order=order, path=cache, reps=2, workload="test")
        assert set(res) == set(autotune.keys_for(n, order))
        for key, (best, times) in res.items():
            assert best in times and all(t > 0 for t in times.values())
        step()
        c.synchronize()
        E1 = E.cpu().numpy()
        tuned = {k: c.get_tuning(k) for k in res}
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), mesh.min, mesh.max, mesh.delta, GAMMA)
    rho, _ = oracle.deposit_particles(x, y, z, om, total_charge=1e-9, resize_mesh=False)
    ef, _ = oracle.space_charge_3d(om, rho)
    E0, _, _ = oracle.interpolate_field(om, ef, x, y, z)
    assert field_err(E1, E0)[0] <= 1e-5
    with osc.Context(0) as c2:
        applied = autotune.apply(c2, path=cache)
        assert set(applied) == set(res)
        assert {k: c2.get_tuning(k) for k in res} == tuned


def test_invalid_tuning_is_rejected():
    with osc.Context(0) as c:
        with pytest.raises(osc.OscError):
            c.set_tuning("gather_run", 5)
        with pytest.raises(osc.OscError):
            c.set_tuning("no_such_key", 1)
        c.set_tuning("gather_run", 8)
        assert c.get_tuning("gather_run") == 8
        c.set_tuning("gather_run", 0)
        assert c.get_tuning("gather_run") == 0
