"""Field reads through the process-wide pool of pinned staging buffers
(transfer.cpp): several handles reading at once from several threads each
borrow a stage of their own, and every read equals the same read done alone.
The reads are large enough (more than one 16 MiB chunk) to run the chunked,
double-buffered path and the multi-threaded host copy."""
import threading

import numpy as np
import pytest

from helpers import spheres

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def test_concurrent_field_reads_match_single_reads(L):
    masks = [spheres((128, 128, 128), 0.45, 4.0, seed=s) for s in (3, 4, 5)]
    solvers = [L.SinglePhase(m, 0.1, (1e-5, 0.0, 0.0), precision="f32") for m in masks]
    try:
        for i, s in enumerate(solvers):
            s.step(10 + 5 * i)
        alone = [s.fields() for s in solvers]
        assert alone[0][1].nbytes > (16 << 20)  # u spans several staging chunks
        out = [[None] * 3 for _ in solvers]
        errors = []

        def read(i):
            try:
                for r in range(3):
                    out[i][r] = solvers[i].fields()
            except Exception as e:  # surfaced below
                errors.append(e)

        threads = [threading.Thread(target=read, args=(i,)) for i in range(len(solvers))]
        for t in threads:
            t.start()
        for t in threads:
            t.join(timeout=300)
        assert not errors, errors
        for i in range(len(solvers)):
            for r in range(3):
                rho, u = out[i][r]
                assert np.array_equal(rho, alone[i][0]) and np.array_equal(u, alone[i][1]), (i, r)
    finally:
        for s in solvers:
            s.close()


def test_populations_read_matches_fields(L):
    """A population read (152 B per node, several chunks) after field reads
    reuses the pooled stage; rho from the populations equals the field rho
    to FP32 storage precision."""
    m = spheres((128, 128, 128), 0.4, 4.0, seed=9)
    with L.SinglePhase(m, 0.1, (1e-5, 0.0, 0.0), precision="f32") as s:
        s.step(20)
        rho, _ = s.fields()
        f = s.populations().reshape(-1, 19)
        assert f.nbytes > (16 << 20)
        assert np.abs(f[1:].sum(axis=1) - rho[1:]).max() < 1e-5


def test_pooled_device_memory_is_reused_and_released(L):
    """A solver created after another one was destroyed takes its memory
    from the process's pool (same results), and lbm_release_cached_memory
    hands the cache back to the driver."""
    import torch

    m = spheres((96, 96, 96), 0.4, 4.0, seed=12)
    out = []
    for _ in range(2):
        with L.SinglePhase(m, 0.1, (1e-5, 0.0, 0.0), precision="f32") as s:
            s.step(30)
            out.append(s.fields())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    free_cached = torch.cuda.mem_get_info()[0]
    L.release_cached_memory()
    assert torch.cuda.mem_get_info()[0] >= free_cached
