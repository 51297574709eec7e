"""GPU tests of geometry paging (nomad_paging_*): per-object BLAS nodes and triangle records
streamed from pinned host memory into a device pool.

Once every wanted object is Resident, traversal and rendering must equal the same scene uploaded
whole with the same residency (bit for bit), which in turn equals the oracle under that residency;
objects that are wanted but not yet Resident are skipped; evicted pool space is reused; onloads
are capped per update and denied past the pool.
"""
import numpy as np
import pytest

from tests import raysets

pytestmark = pytest.mark.gpu


def _rays(sb, seed=5):
    return np.concatenate([raysets.aimed_rays(sb, 6000, seed), raysets.random_rays(sb, 6000, seed + 1)])


def _masked(nb, sb, active_objs, rays, views=None, prim_off=()):
    """Hits (and images) of the whole scene with only `active_objs` resident, traced by the CUDA
    path without paging and checked against the oracle under the same residency (instance
    records with blasRoot = -1 for the evicted objects, activeMask 0 for the primitives off):
    hits bit for bit, images within the path tracer's bar."""
    from oracle import oracle as orc

    active_objs = np.asarray(active_objs, bool)
    ctx = nb.Context()
    try:
        ctx.upload(sb)
        for o in np.nonzero(~active_objs)[0]:
            ctx.set_object_active(int(o), False)
        for p in prim_off:
            ctx.set_primitive_active(int(p), False)
        ctx.flush()
        hits = ctx.trace_closest(rays)
        imgs = ctx.render(views) if views is not None else None
    finally:
        ctx.close()
    active = np.ones(sb.prim_count, np.uint8)
    active[np.asarray(prim_off, np.int64)] = 0
    root = np.ascontiguousarray(sb.instances["blas_root_index"], np.int32).copy()
    root[~active_objs] = -1
    os_ = orc.OracleScene(sb, active=active, blas_root=root)
    want = os_.closest(rays, orc.MODE_REFERENCE_ORDER)
    assert np.array_equal(_bits(hits), _bits(want)), "CUDA path differs from the oracle under this residency"
    if views is not None:
        ref, _, _ = orc.render(os_, sb.materials, views)
        got = np.concatenate([i.reshape(-1, 3) for i in imgs])
        exact = (got == ref).all(1).mean()
        err = (np.abs(got - ref).sum(1) / np.maximum(np.abs(ref).sum(1), 1e-6)).mean()
        assert exact > 0.99 and err < 1e-4, (exact, err)
    return hits, imgs


def _bits(h):
    return np.ascontiguousarray(h).view(np.int32).reshape(-1, 5)


def _full_bytes(nb, sb, width):
    """Bytes of every object's paged nodes and records (the pool that holds the whole scene)."""
    ctx = nb.Context()
    try:
        ctx.upload(sb)
        ctx.paging_enable(1 << 40, width=width)
        return ctx.paging_stats()["full_bytes"]
    finally:
        ctx.close()


def _paged(nb, sb, width, pool_bytes, max_onloads=0):
    ctx = nb.Context()
    ctx.upload(sb)
    ctx.paging_enable(pool_bytes, width=width, max_onloads=max_onloads)
    return ctx


@pytest.mark.parametrize("width", [2, 4, 8])
def test_full_pool_pages_everything_in(nb, small_city, width):
    _, sb = small_city
    rays = _rays(sb)
    ctx = _paged(nb, sb, width, 1 << 40)
    try:
        st = ctx.paging_stats()
        assert st["pool_bytes"] == st["full_bytes"]
        assert (ctx.trace_closest(rays)["inst"] < 0).all()  # nothing streamed yet
        ctx.paging_update()
        st = ctx.paging_stats()
        nonempty = int((sb.instances["primitive_count"] > 0).sum())
        assert st["onloads"] == min(32, nonempty)
        assert st["deferred"] == nonempty - st["onloads"]
        for _ in range(50):
            ctx.paging_wait()
            ctx.paging_update()
            if ctx.paging_stats()["resident"] == nonempty:
                break
        st = ctx.paging_stats()
        assert st["resident"] == nonempty and st["cold"] == sb.object_count - nonempty
        assert st["used_bytes"] == st["full_bytes"] and st["denied"] == 0
        got = ctx.trace_closest(rays)
    finally:
        ctx.close()
    want, _ = _masked(nb, sb, np.ones(sb.object_count, bool), rays)
    assert np.array_equal(_bits(got), _bits(want))


@pytest.mark.parametrize("width", [2, 4])
def test_budgeted_pool_evicts_and_reuses(nb, small_city, width):
    _, sb = small_city
    rays = _rays(sb, 9)
    rng = np.random.default_rng(width)
    n = sb.object_count
    sets = [rng.random(n) < 0.4, rng.random(n) < 0.4, rng.random(n) < 0.4]
    share = max(sb.instances["primitive_count"][s].sum() for s in sets) / sb.prim_count
    pool = int(_full_bytes(nb, sb, width) * min(0.9, share * 1.6))
    ctx = nb.Context()
    ctx.upload(sb)
    ctx.paging_enable(pool, width=width)
    try:
        for k, act in enumerate(sets):
            for o in range(n):
                ctx.set_object_active(o, bool(act[o]))
            ctx.flush()
            for _ in range(100):
                ctx.paging_update()
                ctx.paging_wait()
                states = ctx.paging_states()
                if ((states == 2) == act).all():
                    break
            states = ctx.paging_states()
            assert ((states == 2) == act).all(), (k, ctx.paging_stats())
            st = ctx.paging_stats()
            assert st["used_bytes"] <= st["pool_bytes"] < st["full_bytes"]
            got = ctx.trace_closest(rays)
            want, _ = _masked(nb, sb, act, rays)
            assert np.array_equal(_bits(got), _bits(want)), k
        assert ctx.paging_stats()["evictions"] > 0
    finally:
        ctx.close()


def test_small_pool_denies_onloads(nb, small_city):
    """Objects that do not fit are denied and stay invisible; what is resident traces exactly."""
    _, sb = small_city
    rays = _rays(sb, 13)
    pool = int(_full_bytes(nb, sb, 4) * 0.3)
    ctx = nb.Context()
    ctx.upload(sb)
    ctx.paging_enable(pool, width=4)
    try:
        for _ in range(10):
            ctx.paging_update()
            ctx.paging_wait()
        st = ctx.paging_stats()
        assert st["denied"] > 0 and st["resident"] > 0
        states = ctx.paging_states()
        got = ctx.trace_closest(rays)
    finally:
        ctx.close()
    want, _ = _masked(nb, sb, states == 2, rays)
    assert np.array_equal(_bits(got), _bits(want))


def test_primitive_toggles_follow_pages(nb, small_city):
    """Primitive activity set while an object is Resident, Cached (unlinked, pool copy kept) or
    Cold (never streamed in) reaches the copy that is traced once it is wanted again."""
    _, sb = small_city
    rays = _rays(sb, 17)
    rng = np.random.default_rng(1)
    off = rng.choice(sb.prim_count, size=sb.prim_count // 5, replace=False)
    by_size = np.argsort(-sb.instances["primitive_count"])
    cold_obj, cache_obj = int(by_size[0]), int(by_size[1])
    ctx = _paged(nb, sb, 4, 1 << 40)
    try:
        ctx.set_object_active(cold_obj, False)  # before any update: never streamed in
        ctx.flush()
        for _ in range(10):
            ctx.paging_update()
            ctx.paging_wait()
        ctx.set_object_active(cache_obj, False)
        ctx.flush()
        for _ in range(3):
            ctx.paging_update()
            ctx.paging_wait()
        st = ctx.paging_states()
        assert st[cold_obj] == nb.native.PAGE_COLD and st[cache_obj] == nb.native.PAGE_CACHED
        assert (sb.prim_object[off] == cold_obj).any() and (sb.prim_object[off] == cache_obj).any()
        for p in off:
            ctx.set_primitive_active(int(p), False)
        ctx.flush()
        ctx.set_object_active(cold_obj, True)
        ctx.set_object_active(cache_obj, True)
        # the object toggles re-activated their primitives: switch the chosen ones off again
        for p in off[(sb.prim_object[off] == cold_obj) | (sb.prim_object[off] == cache_obj)]:
            ctx.set_primitive_active(int(p), False)
        ctx.flush()
        for _ in range(10):
            ctx.paging_update()
            ctx.paging_wait()
        assert (ctx.paging_states()[sb.instances["primitive_count"] > 0] == nb.native.PAGE_RESIDENT).all()
        assert ctx.paging_stats()["relinks"] >= 1
        got = ctx.trace_closest(rays)
    finally:
        ctx.close()
    want, _ = _masked(nb, sb, np.ones(sb.object_count, bool), rays, prim_off=off)
    assert np.array_equal(_bits(got), _bits(want))


def test_paged_render_matches_whole_scene(nb, small_city):
    _, sb = small_city
    views = nb.view_pinhole((0, 60, -180), (0, 0, 0), width=160, height=90, spp=2, max_depth=3, seed=4)
    act = np.random.default_rng(3).random(sb.object_count) < 0.6
    ctx = nb.Context()
    ctx.upload(sb)
    ctx.paging_enable(int(ctx.object_bytes().sum()), width=4)
    try:
        for o in np.nonzero(~act)[0]:
            ctx.set_object_active(int(o), False)
        ctx.flush()
        for _ in range(10):
            ctx.paging_update()
            ctx.paging_wait()
        got = ctx.render(views)[0]
    finally:
        ctx.close()
    _, imgs = _masked(nb, sb, act, _rays(sb)[:16], views=views)
    assert np.array_equal(got.view(np.int32), imgs[0].view(np.int32))


def test_device_residency_step_drives_paging(nb, small_city):
    """Ray-hit residency at 40 % of the geometry bytes decides; paging follows the device flags."""
    _, sb = small_city
    rays = _rays(sb, 21)
    ctx = nb.Context()
    ctx.upload(sb)
    nbytes = ctx.object_bytes()
    budget = int(nbytes.sum() * 0.4)
    ctx.paging_enable(int(budget * 1.25), width=4)
    prm = nb.ResidencyParams.make(nb.POLICY_RAYHIT_BUDGET, budget_bytes=budget)
    try:
        for frame in range(12):
            ang = frame * 0.3
            view = nb.view_pinhole((180 * np.sin(ang), 60, -180 * np.cos(ang)), (0, 0, 0), width=96, height=54,
                                   spp=2, max_depth=2, seed=frame)
            ctx.render(view, count_hits=True)
            ctx.residency_step(prm, view, toggles=False)
            ctx.paging_update()
        for _ in range(20):
            ctx.paging_update()
            ctx.paging_wait()
        flags = ctx.residency_flags().astype(bool)
        states = ctx.paging_states()
        assert ((states == 2) == (flags & (sb.instances["primitive_count"] > 0))).all()
        got = ctx.trace_closest(rays)
    finally:
        ctx.close()
    want, _ = _masked(nb, sb, flags, rays)
    assert np.array_equal(_bits(got), _bits(want))


def test_sync_publish_repeats_exactly(nb, small_city):
    """With nomad_paging_set_sync, each update publishes what the previous ones started, so two
    contexts given the same calls go through the same paging states, statistics and images frame
    by frame, however fast their copies ran. A small pool (35 % of the geometry bytes), a ray-hit
    budget of 30 % and 8 onloads per update keep objects streaming, cached and evicted."""
    _, sb = small_city
    runs = []
    for _ in range(2):
        ctx = nb.Context()
        ctx.upload(sb)
        nbytes = ctx.object_bytes()
        ctx.paging_enable(int(nbytes.sum() * 0.35), width=4, max_onloads=8)
        ctx.paging_set_sync(True)
        prm = nb.ResidencyParams.make(nb.POLICY_RAYHIT_BUDGET, budget_bytes=int(nbytes.sum() * 0.3),
                                      camera_motion=0.5)
        trace = []
        try:
            for frame in range(16):
                ang = frame * 0.4
                view = nb.view_pinhole((180 * np.sin(ang), 60, -180 * np.cos(ang)), (0, 0, 0), width=96,
                                       height=54, spp=2, max_depth=2, seed=frame)
                img = ctx.render(view, count_hits=True)[0]
                ctx.residency_step(prm, view, toggles=False)
                ctx.paging_update()
                st = ctx.paging_stats()
                trace.append((ctx.paging_states().copy(), img.copy(),
                              tuple(st[k] for k in ("onloads", "evictions", "deferred", "relinks", "cached"))))
        finally:
            ctx.close()
        runs.append(trace)
    for f, (a, b) in enumerate(zip(*runs)):
        assert np.array_equal(a[0], b[0]), f
        assert np.array_equal(a[1], b[1]), f
        assert a[2] == b[2], f
    onloads, evictions, deferred = runs[0][-1][2][:3]
    assert onloads > 0 and evictions + deferred > 0  # the pool was under pressure


def test_paging_refuses_other_layouts(nb, small_city):
    _, sb = small_city
    ctx = _paged(nb, sb, 4, 1 << 40)
    try:
        with pytest.raises(nb.NomadError):
            ctx.set_traversal(width=8, persistent=1, regroup=1)
        with pytest.raises(nb.NomadError):
            ctx.trace_work(_rays(sb)[:64])
        with pytest.raises(nb.NomadError):
            ctx.paging_enable(1 << 30, width=4)
        assert ctx.traversal()["width"] == 4
    finally:
        ctx.close()
