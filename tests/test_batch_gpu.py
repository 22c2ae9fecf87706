"""Batched and served solves on the GPU.

Per-node arithmetic in the pool is the single-domain FP32 kernel's, and each
instance pulls only from its own node range, so:
  * a batch instance after k steps equals the single-domain solver after k
    steps to FP32 round-off (another kernel, other multiply-add contractions);
  * an instance's result (steps, permeability, fields) is identical alone and
    in a mix with other instances (per-instance sums run over its own tiles in
    a fixed order);
  * the server, which admits requests as nodes free up, returns the same
    results as the batch.
Convergence steps agree with the single-domain run_to_convergence within one
check interval (that path sums in a different order).
"""
import numpy as np
import pytest

from helpers import spheres

pytestmark = pytest.mark.gpu

NU, G = 0.1, (1e-5, 0.0, 0.0)


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


@pytest.fixture(scope="module")
def masks():
    return [spheres((20, 18, 16), 0.5, 3.0, seed=1), spheres((33, 29, 31), 0.45, 4.0, seed=2),
            spheres((24, 40, 12), 0.6, 2.5, seed=3), spheres((48, 48, 48), 0.4, 5.0, seed=4)]


def test_batch_instances_equal_single_domain_solver(L, masks):
    steps = 150
    with L.Batch([(m, NU, G) for m in masks], precision="f32") as b:
        res = b.run(tol=1e-300, check_every=50, max_steps=steps)
        for i, m in enumerate(masks):
            assert res[i]["steps"] == steps and res[i]["status"] == -6
            rho_b, u_b = b.fields(i)
            with L.SinglePhase(m, NU, G, precision="f32") as s:
                s.step(steps)
                rho_s, u_s = s.fields()
                d = s.reduce()
            # same per-node arithmetic in a different kernel: the compiler may
            # contract multiply-adds differently, so equal to FP32 round-off
            assert np.abs(u_b - u_s).max() <= 1e-5 * np.abs(u_s).max()
            assert np.abs(rho_b - rho_s).max() <= 1e-6
            np.testing.assert_allclose(res[i]["perm"][0], d["perm"][0], rtol=1e-5)
            assert res[i]["count"] == s.count


def test_batch_alone_equals_in_mix_and_converges_like_single(L, masks):
    tol, every = 1e-4, 50
    with L.Batch([(m, NU, G) for m in masks], precision="f32") as mix:
        rmix = mix.run(tol=tol, check_every=every, max_steps=20000)
        fmix = [mix.fields(i) for i in range(len(masks))]
    for i in (0, 3):
        with L.Batch([(masks[i], NU, G)], precision="f32") as alone:
            r = alone.run(tol=tol, check_every=every, max_steps=20000)[0]
            assert r["status"] == 0 and r["steps"] == rmix[i]["steps"]
            assert r["perm"][0] == rmix[i]["perm"][0] and r["u_ave"] == rmix[i]["u_ave"]
            rho, u = alone.fields(0)
            assert np.array_equal(u, fmix[i][1]) and np.array_equal(rho, fmix[i][0])
        with L.SinglePhase(masks[i], NU, G, precision="f32") as s:
            d = s.run_to_convergence(tol=tol, check_every=every, max_steps=20000)
            assert abs(d["step"] - r["steps"]) <= every
            np.testing.assert_allclose(d["perm"][0], r["perm"][0], rtol=1e-4)


def test_batch_reset_and_autotune_reproduce(L, masks):
    with L.Batch([(m, NU, G) for m in masks[:3]], precision="f32") as b:
        r1 = b.run(tol=1e-4, check_every=50, max_steps=5000)
        t = b.autotune(trial_steps=5)
        assert t["block"] in (128, 256, 512) and t["ordering"] in (0, 2) and t["mlups"] > 0
        r2 = b.run(tol=1e-4, check_every=50, max_steps=5000)
        # the tuned layout may order the nodes differently: the per-node
        # arithmetic is the same, the flux sums run in another order
        for a, c in zip(r1, r2):
            assert a["steps"] == c["steps"]
            np.testing.assert_allclose(c["perm"][0], a["perm"][0], rtol=1e-6)
        b.reset()
        r3 = b.run(tol=1e-4, check_every=50, max_steps=5000)
        assert [x["perm"][0] for x in r3] == [x["perm"][0] for x in r2]
        info = b.info()
        assert info["node_steps"] == sum(x["steps"] * x["count"] for x in r3) and info["last_run_ms"] > 0


def test_batch_fp16_close_to_fp32(L, masks):
    ms = [masks[1], masks[3]]
    with L.Batch([(m, NU, G) for m in ms], precision="f32") as b32, \
            L.Batch([(m, NU, G) for m in ms], precision="f16") as b16:
        r32 = b32.run(tol=1e-30, check_every=100, max_steps=1500)
        r16 = b16.run(tol=1e-30, check_every=100, max_steps=1500)
        for a, c in zip(r32, r16):
            np.testing.assert_allclose(c["perm"][0], a["perm"][0], rtol=1e-2)


@pytest.mark.parametrize("target,policy", [(0, "fifo"), (30000, "fifo"), (30000, "shortest")])
def test_server_continuous_batching_matches_batch(L, masks, target, policy):
    tol, every = 1e-4, 50
    with L.Batch([(m, NU, G) for m in masks], precision="f32") as b:
        want = b.run(tol=tol, check_every=every, max_steps=20000)
    # a pool that holds the biggest request but not all of them at once
    big = max(int((m == 0).sum()) for m in masks)
    with L.Server(capacity_nodes=big + 2048, max_active=3, precision="f32", tol=tol, check_every=every,
                  max_steps=20000, target_active_nodes=target, policy=policy) as srv:
        ids = [srv.submit(m, NU, G) for m in masks]
        got, rounds, saw_queue = {}, 0, False
        while len(got) < len(masks):
            active, queued = srv.pump()
            saw_queue |= queued > 0 and active > 0
            for r in srv.poll():
                got[r["request_id"]] = r
            rounds += 1
            assert rounds < 5000
        assert saw_queue, "requests should have waited for pool memory"
        for i, rid in enumerate(ids):
            r = got[rid]
            assert r["status"] == 0 and r["steps"] == want[i]["steps"] and r["perm"][0] == want[i]["perm"][0]
            assert r["t_submit"] <= r["t_admit"] <= r["t_done"]
        if policy == "shortest":
            # admitted in ascending estimated work (cells x nx^2), not in
            # arrival order: [0, 2, 1, 3] for these masks
            work = [m.size * m.shape[2] ** 2 for m in masks]
            admitted = [ids.index(r["request_id"]) for r in sorted(got.values(), key=lambda r: r["t_admit"])]
            assert admitted == [int(i) for i in np.argsort(work)] and admitted != sorted(admitted)


def test_server_rejects_oversized_and_bad_requests(L, masks):
    with L.Server(capacity_nodes=4096, max_active=2) as srv:
        with pytest.raises(L.LbmError) as e:
            srv.submit(masks[3], NU, G)
        assert e.value.status == -1
        with pytest.raises(L.LbmError):
            srv.submit(np.ones((4, 4, 4), dtype=np.uint8), NU, G)
        rid = srv.submit(masks[0][:8, :8, :8].copy(), NU, G)
        assert rid > 0
