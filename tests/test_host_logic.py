"""Host-side logic that needs no GPU: workload generators (seeded, shapes
and ranges as specified) and the serving bookkeeping."""
from ct_laboratory_b200.serving import JobSpec, job_bytes, latency_summary
from ct_laboratory_b200.workloads import WORKLOADS


def test_serving_workload_is_seeded_and_in_range():
    w = WORKLOADS["serve"]
    a, b = w.jobs(), w.jobs()
    assert a == b and len(a) == w.n_jobs
    arr = [d["arrival_s"] for d in a]
    assert arr[0] == 0.0 and arr == sorted(arr)
    for d in a:
        assert d["n"] in w.sizes and w.views[0] <= d["views"] <= w.views[1] and w.iters[0] <= d["iters"] <= w.iters[1]
        assert w.I0[0] <= d["I0"] <= w.I0[1] and d["det_nx"] == 2 * d["n"] and d["det_ny"] == 3 * d["n"] // 2


def test_job_footprint_and_latency_summary():
    s = JobSpec(**WORKLOADS["serve"].jobs()[0])
    assert job_bytes(s) == 36 * s.n_ray + 16 * s.n ** 3
    # the fixed-point adjoint's int64 sums count 8 B more per voxel
    assert job_bytes(s, deterministic_adjoint=True) == 36 * s.n_ray + 24 * s.n ** 3
    summ = latency_summary([{"latency_s": 1.0, "arrival_s": 0.0, "finish_s": 1.0},
                            {"latency_s": 3.0, "arrival_s": 1.0, "finish_s": 4.0}])
    assert summ["jobs"] == 2 and abs(summ["jobs_per_s"] - 0.5) < 1e-12 and summ["p50_s"] == 2.0


def test_batch_workload_is_seeded_and_in_range():
    w = WORKLOADS["batch64"]
    ins = w.instances()
    assert ins == w.instances() and len(ins) == 64
    for d in ins:
        assert d["side"] in w.sides and abs(d["pixel"] * d["side"] - w.fov) < 1e-9
        if d["kind"] == "ring":
            assert w.sources[0] <= d["sources"] <= w.sources[1] and d["views"] == d["sources"] * d["frames"]
        else:
            assert w.views[0] <= d["views"] <= w.views[1]


def test_projector_module_copies_without_its_tile_lists():
    """A 3-D projector module deep-copies and pickles; its cached
    active-tile lists (device state) are left behind and rebuilt on use."""
    import copy
    import pickle

    import torch

    from ct_laboratory_b200 import _native as N
    from ct_laboratory_b200.tomography import CTProjector3DModule
    src = torch.zeros(4, 3)
    dst = torch.ones(4, 3)
    m = CTProjector3DModule(2, 2, 2, torch.eye(3), torch.zeros(3), src, dst, device=torch.device("cpu"))
    opts = N.ActiveRayOpts()
    opts.active = (torch.zeros(3, dtype=torch.int32), 3)
    m._active[("key",)] = ((m.src, m.dst, m.M, m.b), (0,), opts)
    for c in (copy.deepcopy(m), pickle.loads(pickle.dumps(m))):
        assert c._active == {} and torch.equal(c.src, m.src)
    assert len(m._active) == 1


def test_bare_call_tile_cache_keys(monkeypatch):
    """The active-tile cache of bare _C calls hits only for the same geometry
    tensors at the same versions with the same M^-1 and b values: a fresh
    M^-1 tensor with equal values hits; changed values, an in-place edit of
    the rays or a new ray tensor miss.  (The device work of the list is
    replaced by a counter here.)"""
    import torch

    from ct_laboratory_b200 import _C
    from ct_laboratory_b200 import _native as N
    calls = []

    def fake(t, src, dst, M_inv, b, dims):
        calls.append(1)
        return ("list", len(calls))

    monkeypatch.setattr(N, "active_tiling", fake)
    _C._BARE_TILES.clear()
    t = N.tiling(2, 32, 4, 128, 4, 1, tile_rows=32, block_threads=128)
    src, dst = torch.rand(256, 3), torch.rand(256, 3)
    Mi, b = torch.eye(3), torch.zeros(3)
    first = _C._bare_active(t, src, dst, Mi, b, (8, 8, 8))
    assert _C._bare_active(t, src, dst, torch.eye(3), b.clone(), (8, 8, 8)) is first and len(calls) == 1
    assert _C._bare_active(t, src, dst, Mi, b + 1.0, (8, 8, 8)) != first and len(calls) == 2
    src.add_(0.0)  # an in-place edit bumps the version
    assert len(calls) == 2 and _C._bare_active(t, src, dst, Mi, b + 1.0, (8, 8, 8)) and len(calls) == 3
    other = src.clone()
    _C._bare_active(t, other, dst, Mi, b + 1.0, (8, 8, 8))
    assert len(calls) == 4
    assert _C._bare_active(None, src, dst, Mi, b, (8, 8, 8)) is None
    assert _C._bare_active(N.flat_opts(), src, dst, Mi, b, (8, 8, 8)).n_view == 0  # flat launches carry no list
    _C._BARE_TILES.clear()
