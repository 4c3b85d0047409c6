"""The allocation-free record sum (lbm_record_forces_noalloc) against the
force and moment lbm_run returns for the same step.

Callers that cannot allocate device memory at the point of use (a host whose
device memory belongs to its own pool allocator, an embedded caller with a
fixed footprint, a loop that cannot afford cudaMalloc/cudaFree) call this
entry point with device pointers only.  The test puts a lattice's wall
records into device memory, calls the entry point twice in a row through the
C ABI and compares each result with lbm_run's force and moment of the step
the records come from (FP64 sums of the same float words, so to 1e-12).
Collected last so a failure here leaves every other test already run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_record_forces_noalloc_matches_run():
    import torch

    from simlab_b200.cases import sphere_re40
    from simlab_b200.lbm import Lattice, LbmError, Storage, library, record_forces_noalloc

    torch.cuda.set_device(0)
    st, vox = sphere_re40(Storage.FP32, debug_dump=False)
    lat = Lattice(st, vox)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for steps in (37, 11):  # two calls in a row, each on a fresh step's records
        forces = lat.run(steps)
        recs = torch.from_numpy(lat.records().view(np.int32)).to("cuda")
        record_forces_noalloc(recs.data_ptr(), lat.nrec, out.data_ptr(), stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = forces[-1]
        assert np.all(np.isfinite(got))
        assert np.allclose(got, want, rtol=1e-12, atol=1e-14 * np.max(np.abs(want))), (got, want)
    # more records than the fixed scratch holds is refused, nothing launched
    big = library().lbm_record_forces_noalloc_max() + 1
    with pytest.raises(LbmError, match="too many records"):
        record_forces_noalloc(recs.data_ptr(), big, out.data_ptr(), stream)
    lat.close()
