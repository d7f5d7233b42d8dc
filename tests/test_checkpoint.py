"""Checkpoint / pickup files (Write_Model2D / Read_Model2D layout) on CPU:
round trips of host arrays and attributes, element slabs, error paths, and the
reference's TimeStamp."""
import numpy as np
import pytest


def test_round_trip_arrays_attributes_and_slabs(tmp_path):
    from self_b200.checkpoint import Checkpoint
    rng = np.random.default_rng(0)
    P, nVar, nEl = 4, 3, 7
    sol = np.asfortranarray(rng.normal(size=(P, P, nVar, nEl)))
    ids = np.asfortranarray(rng.integers(-5, 5, size=(5, 4, nEl)).astype(np.int32))
    f32 = np.asfortranarray(rng.normal(size=(6, 2)).astype(np.float32))
    path = tmp_path / "a.ckpt"
    with Checkpoint(path, "w") as c:
        c.attr("N", 3)
        c.attr("time", 1.25)
        c.put("/state/interior/solution", sol)
        c.put("/mesh/sideInfo", ids)
        c.put("/other", f32)
    with Checkpoint(path, "r") as c:
        assert c.attr("N") == 3 and c.attr("time") == 1.25
        assert c.info("/state/interior/solution") == (1, [P, P, nVar, nEl])
        np.testing.assert_array_equal(c.get("/state/interior/solution"), sol)
        np.testing.assert_array_equal(c.get("/mesh/sideInfo"), ids)
        np.testing.assert_array_equal(c.get("/other"), f32)
        # a rank's element slab, as Read_Model2D reads with MPI
        np.testing.assert_array_equal(c.get("/state/interior/solution", 2, 3), sol[..., 2:5])


def test_error_paths(tmp_path):
    from self_b200._lib import SelfGpuError
    from self_b200.checkpoint import Checkpoint
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(b"not a checkpoint file")
    with pytest.raises(SelfGpuError):
        Checkpoint(bad, "r")
    path = tmp_path / "b.ckpt"
    with Checkpoint(path, "w") as c:
        c.put("/x", np.zeros((2, 3)))
    with Checkpoint(path, "r") as c:
        with pytest.raises(SelfGpuError):
            c.get("/missing")
        with pytest.raises(SelfGpuError):
            c.get("/x", 2, 2)  # slab outside the element range
        with pytest.raises(SelfGpuError):
            c.attr("N")
    data = path.read_bytes()
    trunc = tmp_path / "t.ckpt"
    trunc.write_bytes(data[:-5])
    with pytest.raises(SelfGpuError):
        Checkpoint(trunc, "r")
    with pytest.raises(SelfGpuError):
        Checkpoint(tmp_path / "no_such_dir" / "x.ckpt", "w")


@pytest.mark.parametrize("t,stamp", [(0.0, "0000000000000"), (1.5, "0000000001500"), (61.25, "0000000101250"),
                                     (3723.004, "0000010203004"), (90061.999, "0001010101999"),
                                     (59.9996, "0000000100000")])
def test_time_stamp_follows_the_reference(t, stamp):
    """DDDDHHMMSSmmm with NINT milliseconds and carries (src/SELF_SupportRoutines.f90:856-924)."""
    from self_b200.checkpoint import time_stamp
    assert time_stamp(t) == stamp
