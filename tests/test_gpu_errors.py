"""Error paths that need a device: a plan larger than the device reports a status
(never an abort), and the device stays usable afterwards."""
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid

pytestmark = pytest.mark.gpu


def test_plan_larger_than_the_device_reports_out_of_memory():
    # 400000^2 FP64 cells: a 1.28 TB workspace, far beyond the device's memory
    with pytest.raises(ffs.FFSError) as e:
        ffs.Plan(2, "Box2D9P", (400000, 400000), 8, boundary="fixed")
    assert e.value.status == ffs.ERR_OUT_OF_MEMORY, str(e.value)
    plan = ffs.Plan(2, "Box2D9P", (64, 48), 3, boundary="fixed")
    x = seeded_grid((48, 64), 1)
    ref = oracle.run(x, ffs.shape_info("Box2D9P").weights, 1, 3, oracle.FIXED)
    assert rel_errors(plan.run_host(x), ref)[0] <= 1e-12
