"""Asynchronous snapshot output of a device-resident run: the snapshots on
disk are the states the run produced, in order, although the run goes on
(and overwrites its buffers) while the copies and the file writes are in
flight."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_async_snapshots_of_a_running_integration(tmp_path):
    from suetes_b200 import StateRing
    from suetes_b200.output import AsyncSnapshotWriter, NetcdfSnapshots, SimulationOutputWriter
    from suetes_b200.workloads import rising_bubble
    st, s0, _ = rising_bubble(24, 20, 16, dtype=torch.float32, solver_tol=1e-6, solver_maxiter=30,
                              solver_restart=20)
    ds = st.to_device_state(s0)
    path = str(tmp_path / "bubble.nc")
    aw = AsyncSnapshotWriter(SimulationOutputWriter(path, st.physics.grid, ["u", "w", "th_p"]), depth=2)
    ring = StateRing(ds.core)
    cur, expect = ds, []
    for n in range(5):
        nxt = ring.next_output(cur)
        st.step_device(cur, nxt, None)
        cur = nxt
        aw.submit({"u": cur.t["u"], "w": cur.t["w"], "th_p": cur.t["th_p"]}, t_seconds=float(n))
        torch.cuda.synchronize()
        expect.append({k: cur.t[k].cpu().numpy().copy() for k in ("u", "w", "th_p")})
    aw.close()
    rd = NetcdfSnapshots(path)
    try:
        assert len(rd) == 5 and list(rd.times) == [0.0, 1.0, 2.0, 3.0, 4.0]
        for n in range(5):
            for k in ("u", "w", "th_p"):
                np.testing.assert_array_equal(rd[n][k], expect[n][k])
    finally:
        rd.close()
