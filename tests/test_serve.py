"""Serving (vrt_server_*): requests of several sessions, with voxel edits
between frames, are batched continuously; each request's image must equal the
image of the same request sequence rendered alone, session by session."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SESSIONS = [(2, 128, 11, 320, 180, 2), (1, 64, 1, 256, 144, 3), (3, 128, 4, 200, 112, 1), (2, 256, 2, 480, 270, 2)]


@pytest.fixture(scope="module")
def ctx(vrt):
    c = vrt.Context(0)
    yield c
    c.close()


def _requests(vrt, spawns, n_req, seed):
    rng = np.random.default_rng(seed)
    frames = [0] * len(SESSIONS)
    reqs = []
    for _ in range(n_req):
        k = int(rng.integers(0, len(SESSIONS)))
        kind, n, sd, W, H, nb = SESSIONS[k]
        f = frames[k]
        frames[k] += 1
        pose = vrt.camera_spline(spawns[k], f)
        prev = vrt.camera_spline(spawns[k], f - 1) if f else None
        u = vrt.make_uniforms(pose, prev, vrt.Lighting(), 7 + f, nb, 3, W, H)
        size = rng.integers(1, 17, 3)
        lo = rng.integers(0, n - 16, 3)
        val = 0 if rng.random() < 0.5 else int(rng.integers(1, 1 << 24))
        edits = [(int(lo[0]), int(lo[1]), int(lo[2]), int(lo[0] + size[0] - 1), int(lo[1] + size[1] - 1),
                  int(lo[2] + size[2] - 1), val)]
        reqs.append((k, u, edits))
    return reqs


def test_server_results_equal_alone(ctx, vrt):
    vox, spawns, served, ref_sc, ref_s, srv_sc = [], [], [], [], [], []
    for kind, n, sd, W, H, nb in SESSIONS:
        v, sp = vrt.generate_scene(kind, n, sd)
        vox.append(v)
        spawns.append(sp)
        sc = vrt.Scene(ctx, v, n)
        srv_sc.append(sc)
        served.append(vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, path_kernel="batch_only"))
        rsc = vrt.Scene(ctx, v, n)
        ref_sc.append(rsc)
        ref_s.append(vrt.Session(ctx, rsc, W, H, firefly_clamp=10.0))
    reqs = _requests(vrt, spawns, 24, 3)
    server = vrt.Server(ctx, served, max_in_flight=2)
    outs = []
    tickets = {}
    done = []
    for i, (k, u, edits) in enumerate(reqs):
        W, H = SESSIONS[k][3], SESSIONS[k][4]
        buf = np.zeros(W * H * 4, np.uint8)
        outs.append(buf)
        tickets[server.submit(k, u, edits, ldr_out=buf)] = i
        if i % 5 == 4:
            done += server.poll()             # requests keep arriving while batches run
    done += server.drain()
    assert sorted(tickets) == sorted(t for t, *_ in done)
    for t, sess, t_arr, t_done in done:
        assert t_done >= t_arr - 1e-3
    # the same requests, session by session, through plain frames
    for i, (k, u, edits) in enumerate(reqs):
        for e in edits:
            ref_sc[k].edit_box(*e)
        ref_s[k].frame(u)
        want = ref_s[k].ldr().ravel()
        assert np.array_equal(outs[i], want), f"request {i} (session {k}) differs"
    for k in range(len(SESSIONS)):
        assert np.array_equal(served[k].accum(), ref_s[k].accum())
        v1, b1, m1 = srv_sc[k].read()
        v2, b2, m2 = ref_sc[k].read()
        assert np.array_equal(v1, v2) and np.array_equal(b1, b2) and np.array_equal(m1, m2)
    server.close()
    for s in served + ref_s:
        s.close()
    for sc in srv_sc + ref_sc:
        sc.close()


def test_server_admission_budget(vrt):
    c = vrt.Context(0, hbm_budget_bytes=64 << 20)
    vox, _ = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(c, vox, 64)
    ok = [vrt.Session(c, sc, 640, 360, path_kernel="batch_only")]
    with pytest.raises(vrt.VrtError) as e:
        for _ in range(8):
            ok.append(vrt.Session(c, sc, 640, 360, path_kernel="batch_only"))
    assert e.value.code == 5
    for s in ok:
        s.close()
    sc.close()
    c.close()


def _session_bytes(vrt, W, H):
    """Device bytes of a batch-only session (measured on a scratch context)."""
    c = vrt.Context(0)
    vox, _ = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(c, vox, 64)
    b0 = c.bytes_in_use
    s = vrt.Session(c, sc, W, H, firefly_clamp=10.0, path_kernel="batch_only")
    b = c.bytes_in_use - b0
    s.close()
    sc.close()
    c.close()
    return b


def test_dynamic_server_admission_queue(vrt):
    """Sessions that do not fit the HBM budget wait in the admission queue and
    are admitted, in arrival order, as soon as a close returns their memory;
    requests of the admitted sessions render what they render alone."""
    W, H = 320, 180
    per = _session_bytes(vrt, W, H)
    vox, spawn = vrt.generate_scene(1, 64, 1)
    probe = vrt.Context(0)
    psc = vrt.Scene(probe, vox, 64)
    scene_bytes = probe.bytes_in_use
    psc.close()
    probe.close()
    # budget: the scene, the server's pool for 2 sessions and room for exactly 2 sessions
    pool = 2 * W * H
    c0 = vrt.Context(0)
    s0 = vrt.Server(c0, None, max_in_flight=2, max_sessions=4, max_pixels=pool)
    pool_bytes = c0.bytes_in_use
    s0.close()
    c0.close()
    ctx = vrt.Context(0, hbm_budget_bytes=scene_bytes + pool_bytes + 2 * per + per // 2)
    sc = vrt.Scene(ctx, vox, 64)
    srv = vrt.Server(ctx, None, max_in_flight=2, max_sessions=4, max_pixels=pool)
    t = [srv.open_session(sc, W, H, firefly_clamp=10.0) for _ in range(4)]
    slots = [srv.session_of(x) for x in t]
    assert slots[0] is not None and slots[1] is not None and slots[2] is None and slots[3] is None
    assert srv.session_counts() == (2, 2)
    # frames on the two open sessions, then close the first: the third is admitted
    outs = {}
    for f in range(3):
        for k in (0, 1):
            u = vrt.make_uniforms(vrt.camera_spline(spawn, f + k), None, vrt.Lighting(), 40 + f, 2, 3, W, H)
            buf = np.zeros(W * H * 4, np.uint8)
            outs[(k, f)] = (u, buf)
            srv.submit(slots[k], u, ldr_out=buf)
    srv.close_session(slots[0])
    assert srv.session_of(t[2]) is None          # its session still has requests queued
    srv.drain()
    srv.poll()
    s2 = srv.session_of(t[2])
    assert s2 is not None and srv.session_of(t[3]) is None
    assert srv.session_counts() == (2, 1)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 77, 2, 3, W, H)
    buf = np.zeros(W * H * 4, np.uint8)
    srv.submit(s2, u, ldr_out=buf)
    srv.drain()
    # alone: the same request sequences on fresh sessions of an unlimited context
    ref = vrt.Context(0)
    rsc = vrt.Scene(ref, vox, 64)
    for k in (0, 1):
        rs = vrt.Session(ref, rsc, W, H, firefly_clamp=10.0)
        for f in range(3):
            uu, b = outs[(k, f)]
            rs.frame(uu)
            assert np.array_equal(b, rs.ldr().ravel()), (k, f)
        rs.close()
    rs = vrt.Session(ref, rsc, W, H, firefly_clamp=10.0)
    rs.frame(u)
    assert np.array_equal(buf, rs.ldr().ravel())
    rs.close()
    rsc.close()
    ref.close()
    srv.close()
    sc.close()
    ctx.close()


def test_sequential_server_equals_alone(ctx, vrt):
    """The unbatched form the batched server is measured against: requests one
    after another through each session's own frame path."""
    vox, spawns, served, ref_sc, ref_s, srv_sc = [], [], [], [], [], []
    for kind, n, sd, W, H, nb in SESSIONS:
        v, sp = vrt.generate_scene(kind, n, sd)
        spawns.append(sp)
        sc = vrt.Scene(ctx, v, n)
        srv_sc.append(sc)
        served.append(vrt.Session(ctx, sc, W, H, firefly_clamp=10.0))
        rsc = vrt.Scene(ctx, v, n)
        ref_sc.append(rsc)
        ref_s.append(vrt.Session(ctx, rsc, W, H, firefly_clamp=10.0))
    reqs = _requests(vrt, spawns, 12, 9)
    server = vrt.Server(ctx, served, max_in_flight=2)
    server.set_sequential(True)
    outs = []
    for k, u, edits in reqs:
        W, H = SESSIONS[k][3], SESSIONS[k][4]
        buf = np.zeros(W * H * 4, np.uint8)
        outs.append(buf)
        server.submit(k, u, edits, ldr_out=buf)
    done = server.drain()
    assert len(done) == len(reqs)
    for i, (k, u, edits) in enumerate(reqs):
        for e in edits:
            ref_sc[k].edit_box(*e)
        ref_s[k].frame(u)
        assert np.array_equal(outs[i], ref_s[k].ldr().ravel()), f"request {i}"
    server.close()
    for s in served + ref_s:
        s.close()
    for sc in srv_sc + ref_sc:
        sc.close()


@pytest.mark.parametrize("solo,min_batch", [(300 * 170, 1), (0, 3), (300 * 170, 2)])
def test_hybrid_server_equals_alone(ctx, vrt, solo, min_batch):
    """Large views alone through their own frame path, small ones batched
    (vrt_server_set_solo_pixels), and requests alone while fewer than
    min_batch sessions wait (vrt_server_set_min_batch): every request still
    renders what it renders alone."""
    vox, spawns, served, ref_sc, ref_s, srv_sc = [], [], [], [], [], []
    for kind, n, sd, W, H, nb in SESSIONS:
        v, sp = vrt.generate_scene(kind, n, sd)
        spawns.append(sp)
        sc = vrt.Scene(ctx, v, n)
        srv_sc.append(sc)
        served.append(vrt.Session(ctx, sc, W, H, firefly_clamp=10.0))
        rsc = vrt.Scene(ctx, v, n)
        ref_sc.append(rsc)
        ref_s.append(vrt.Session(ctx, rsc, W, H, firefly_clamp=10.0))
    reqs = _requests(vrt, spawns, 20, 21)
    server = vrt.Server(ctx, served, max_in_flight=2)
    server.set_solo_pixels(solo)            # 300 x 170: the 320x180 and 480x270 views render alone
    server.set_min_batch(min_batch)
    outs = []
    for i, (k, u, edits) in enumerate(reqs):
        W, H = SESSIONS[k][3], SESSIONS[k][4]
        buf = np.zeros(W * H * 4, np.uint8)
        outs.append(buf)
        server.submit(k, u, edits, ldr_out=buf)
        if i % 4 == 3:
            server.poll()
    server.drain()
    for i, (k, u, edits) in enumerate(reqs):
        for e in edits:
            ref_sc[k].edit_box(*e)
        ref_s[k].frame(u)
        assert np.array_equal(outs[i], ref_s[k].ldr().ravel()), f"request {i}"
    server.close()
    for s in served + ref_s:
        s.close()
    for sc in srv_sc + ref_sc:
        sc.close()
