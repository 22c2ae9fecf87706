"""lbm_reduce_noalloc: the diagnostics reduction for callers that cannot
allocate device memory (they own every device buffer and pass it in; the
library's only scratch is a static device array).

Checked against lbm_reduce on the same state, through the C ABI, on two calls
in a row, with the tolerance the FP64 reduction tests use (1e-12 relative:
both sum the same per-node terms, in different tree orders).  Collected last
so that a run stopping at the first failure has run every other test; it also
passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import spheres

pytestmark = pytest.mark.gpu

NU = 0.1
G = (1e-5, 2e-6, -3e-6)


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def diag_from_sums(r, nx, ny, nz, porosity):
    """The lbm_reduce post-processing (Error SP3:3149-3183, Comput_Perm SP3:3611-3638)."""
    V = nx * ny * nz
    out = {"u_rel_change": np.sqrt(r[0]) / (np.sqrt(r[1]) + 1e-30), "u_max": np.sqrt(r[3]),
           "u_mean_speed": r[2] / (V * porosity), "mass": r[7],
           "perm": [r[4 + d] / V * NU / G[d] for d in range(3)]}
    a = np.array(r[4:7]) / (V * porosity)
    out["u_ave"] = float(np.sqrt((a * a).sum()))
    return out


def call_noalloc(L, f_ref_layout, u_prev_ref_layout, count, pad=0):
    """Caller-owned device arrays in the documented layout, f[q][p] and
    u_prev[d][p] with rows of count + pad entries; the padding holds NaN, so
    a kernel that read it would poison every sum.  u_prev_ref_layout None
    passes NULL."""
    import torch

    stride = count + pad

    def rows(a):
        host = np.full((a.shape[1], stride), np.nan)
        host[:, :count] = a[1:].T
        return torch.tensor(host, dtype=torch.float64, device="cuda")

    f_dev = rows(f_ref_layout)
    u_dev = rows(u_prev_ref_layout) if u_prev_ref_layout is not None else None
    out = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = L.lib().lbm_reduce_noalloc(C.c_void_p(f_dev.data_ptr()),
                                   C.c_void_p(u_dev.data_ptr()) if u_dev is not None else None, count, stride,
                                   count - 1, G[0], G[1], G[2], C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert st == 0, L.lib().lbm_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def compare(d_new, d_old):
    for k in ("u_rel_change", "u_max", "u_mean_speed", "u_ave", "mass"):
        np.testing.assert_allclose(d_new[k], d_old[k], rtol=1e-12, err_msg=k)
    np.testing.assert_allclose(d_new["perm"], d_old["perm"], rtol=1e-12)


def test_noalloc_matches_lbm_reduce_on_two_calls(L):
    import torch

    assert torch.cuda.is_available()
    mask = spheres((30, 26, 22), 0.5, 3.0, seed=77)
    nz, ny, nx = mask.shape
    with L.SinglePhase(mask, NU, G, precision="f64") as s:
        results = []
        for steps in (40, 25):  # two calls in a row on different states
            s.step(steps - 1)
            _, u_prev = s.fields()
            s.step(1)
            f = s.populations()
            d_old = s.reduce()
            r = call_noalloc(L, f, u_prev, s.count)
            compare(diag_from_sums(r, nx, ny, nz, s.porosity), d_old)
            results.append(r)
        assert not np.array_equal(results[0], results[1])
        # the same inputs twice give the same sums (scratch fully rewritten)
        r2 = call_noalloc(L, f, u_prev, s.count)
        assert np.array_equal(r2, results[1])


def test_noalloc_padded_rows_and_null_previous_velocity(L):
    """Rows longer than the node count (stride = n + 37, NaN in the padding)
    give lbm_reduce's sums; without u_prev the change sum is exactly zero and
    the other seven sums are unchanged."""
    mask = spheres((26, 22, 30), 0.5, 3.0, seed=78)
    nz, ny, nx = mask.shape
    with L.SinglePhase(mask, NU, G, precision="f64") as s:
        s.step(30)
        _, u_prev = s.fields()
        s.step(1)
        f = s.populations()
        d_old = s.reduce()
        padded = call_noalloc(L, f, u_prev, s.count, pad=37)
        compare(diag_from_sums(padded, nx, ny, nz, s.porosity), d_old)
        tight = call_noalloc(L, f, u_prev, s.count)
        no_prev = call_noalloc(L, f, None, s.count, pad=37)
    assert np.isfinite(padded).all()
    np.testing.assert_allclose(padded, tight, rtol=1e-13)
    assert no_prev[0] == 0.0
    np.testing.assert_allclose(no_prev[1:], padded[1:], rtol=1e-13)


def test_noalloc_rejects_sizes_beyond_its_scratch(L):
    lib = L.lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = lib.lbm_reduce_noalloc(one, None, 16_777_217, 16_777_217, -1, 0.0, 0.0, 0.0, one, None)
    assert st == -1
    assert "exceeds" in lib.lbm_last_error().decode()
    st = lib.lbm_reduce_noalloc(one, None, 100, 50, -1, 0.0, 0.0, 0.0, one, None)
    assert st == -1
