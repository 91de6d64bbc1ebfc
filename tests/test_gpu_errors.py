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


def test_batch_dependency_wait_that_runs_out_reports_a_timeout(monkeypatch):
    """A batch whose dependency waits are bounded to zero polls: the items of pass 2 of a
    four-pass problem are popped while pass 1 is still running, so some wait gives up.
    The kernel records the timeout code in the batch's status word and goes on (every
    access stays inside the problem's buffers); ffs_batch_status returns FFS_ERR_TIMEOUT;
    the device then still solves a grid exactly.  The wait is a bounded poll of a
    global counter, so nothing faults or hangs."""
    import ctypes

    import torch
    monkeypatch.setenv("FFS_BATCH_WAIT_POLLS", "0")
    plan = ffs.Plan(2, "Box2D9P", (2048, 2048), 32, boundary="fixed", form="fp64", tau=8)
    assert plan.info["passes"] == 4
    x = torch.from_numpy(seeded_grid((2048, 2048), 3)).cuda()
    y = torch.empty_like(x)
    batch = ffs.Batch([plan])
    monkeypatch.delenv("FFS_BATCH_WAIT_POLLS")
    batch.execute([x.data_ptr()], [y.data_ptr()], torch.cuda.current_stream().cuda_stream)
    word = ctypes.c_int(0)
    st = ffs.lib.ffs_batch_status(batch._h, ctypes.byref(word))
    assert st == ffs.ERR_TIMEOUT, ffs.lib.ffs_last_error_string().decode()
    assert word.value == 4  # the dependency-wait code
    batch.close()
    # a batch created without the override waits as long as it needs
    batch = ffs.Batch([plan])
    batch.execute([x.data_ptr()], [y.data_ptr()], torch.cuda.current_stream().cuda_stream)
    assert batch.status() == 0
    ref = plan.run(x)
    torch.cuda.synchronize()
    assert rel_errors(y.cpu().numpy(), ref.cpu().numpy())[0] <= 1e-12
    batch.close()
    small = ffs.Plan(2, "Box2D9P", (64, 48), 3, boundary="fixed")
    h = seeded_grid((48, 64), 1)
    ref = oracle.run(h, ffs.shape_info("Box2D9P").weights, 1, 3, oracle.FIXED)
    assert rel_errors(small.run_host(h), ref)[0] <= 1e-12
