"""Population snapshots (flb_snapshot_save / flb_snapshot_restore): checkpoint
and resume.  A run restored from a snapshot continues bit for bit like the run
that never stopped, from device or host buffers, for single- and multi-block
handles; a snapshot of another lattice is rejected."""
import numpy as np
import pytest
import torch

import freelb_b200 as F
from freelb_b200 import geometry as G

pytestmark = pytest.mark.gpu


def resumed_equals_continuous(lat, steps, where):
    n = lat.snapshot_bytes()
    if where == "device":
        buf = torch.empty(n, dtype=torch.uint8, device="cuda:0")
    else:
        buf = torch.empty(n, dtype=torch.uint8).pin_memory()
    lat.step(steps)
    lat.snapshot_save(buf.data_ptr(), n)
    lat.step(steps)
    ref = [lat.download_pops(block=k) for k in range(lat.nblocks)]
    lat.snapshot_restore(buf.data_ptr(), n)
    lat.step(steps)
    for k in range(lat.nblocks):
        assert np.array_equal(lat.download_pops(block=k), ref[k])


@pytest.mark.parametrize("where", ["device", "host"])
@pytest.mark.parametrize("storage,model", [("fp32", "bgk"), ("fp16s", "mrt"), ("fp64", "les"),
                                           ("fp32s", "bgk")])
def test_resume_single_block(gpu_ok, storage, model, where):
    lat = F.cavity(30, tau=0.55, storage=storage, model=model)
    resumed_equals_continuous(lat, 12, where)


def test_resume_blocks_with_halo(gpu_ok):
    ni = 40
    blocks = G.uneven_blocks(ni, edges=(8, 12, 16), seed=3)
    n = ni + 2
    lat = F.Lattice.blocks(G.block_tuples(blocks), 0.55, mode="halo")
    flags = F.cavity_flags(ni)
    u = np.zeros((n ** 3, 3), dtype=np.float32)
    u[flags == 8, 0] = np.float32(0.1)
    for k, b in enumerate(blocks):
        lat.upload_flags(G.slice_block(flags, n, b), block=k)
        lat.upload_field("u", G.slice_block(u, n, b, comps=3), block=k)
    resumed_equals_continuous(lat, 10, "device")


def test_snapshot_of_another_lattice_is_rejected(gpu_ok):
    a = F.cavity(20)
    n = a.snapshot_bytes()
    buf = torch.zeros(n + 64, dtype=torch.uint8, device="cuda:0")
    with pytest.raises(F.FlbError):  # no header yet
        a.snapshot_restore(buf.data_ptr(), n)
    with pytest.raises(F.FlbError):  # buffer too short
        a.snapshot_save(buf.data_ptr(), n - 1)
    a.snapshot_save(buf.data_ptr(), n)
    for other in (F.cavity(20, storage="fp16s"), F.cavity(21)):
        with pytest.raises(F.FlbError):
            other.snapshot_restore(buf.data_ptr(), other.snapshot_bytes())
