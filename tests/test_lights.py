"""Scene lights (scene.js:58-200, 435-461): the emissive-face light list,
its power alias table and the per-brick top-16 light grid.  CPU checks of the
restatement; GPU builds compared with it bit for bit."""
import numpy as np
import pytest


def _one_light_scene(n=16):
    vox = np.zeros((n, n, n), np.uint32)            # [z, y, x]
    vox[5, 5, 5] = 200 | (100 << 8) | (50 << 16) | (120 << 24)     # emissive
    vox[5, 5, 6] = 0x808080                         # solid neighbour on +x
    return vox.ravel()


def test_light_list_faces_and_weight(orc):
    words, w = orc.light_list(_one_light_scene(), 16)
    assert len(words) == 5                          # +x face covered by the neighbour
    faces = sorted(int(x >> 27) for x in words[:, 0])
    assert faces == [1, 2, 3, 4, 5]
    x, y, z = words[0, 0] & 0x1ff, (words[0, 0] >> 9) & 0x1ff, (words[0, 0] >> 18) & 0x1ff
    assert (x, y, z) == (5, 5, 5)
    r, g, b, e = 200 / 255, 100 / 255, 50 / 255, 120 / 255
    assert w[0] == e * ((0.2126 * r) * r + (0.7152 * g) * g + (0.0722 * b) * b)


def test_alias_table_reproduces_distribution(orc):
    wts = np.array([1.0, 2.0, 3.0, 4.0, 0.0, 10.0])
    t = orc.light_alias(wts)
    n = len(wts)
    mass = np.zeros(n)
    for i in range(n):
        mass[i] += t[i, 0] / n
        mass[int(t[i, 1])] += (1 - t[i, 0]) / n
    np.testing.assert_allclose(mass, wts / wts.sum(), atol=1e-6)
    np.testing.assert_allclose(t[:, 2], np.where(wts > 0, wts / wts.sum(), 1 / n), rtol=1e-6)


def test_light_grid_single_light(orc):
    n = 16
    words, w = orc.light_list(_one_light_scene(n), n)
    g = orc.light_grid(n, words, w)
    bg = n // 8
    assert g.shape == (bg ** 3, 34)
    # every cell in front of a face holds that face with weight w / max(d^2, 16)
    for cell in range(bg ** 3):
        bx, by, bz = cell % bg, (cell // bg) % bg, cell // (bg * bg)
        cc = np.array([(bx + 0.5) * 8, (by + 0.5) * 8, (bz + 0.5) * 8])
        expect = []
        for i, (w0, _) in enumerate(words):
            v = np.array([w0 & 0x1ff, (w0 >> 9) & 0x1ff, (w0 >> 18) & 0x1ff], float)
            f = int(w0 >> 27)
            ax, pos = f >> 1, 1 if f % 2 == 0 else 0
            c = v + 0.5
            c[ax] = v[ax] + pos
            nn = np.zeros(3)
            nn[ax] = 1.0 if pos else -1.0
            d = cc - c
            if d @ nn <= 0:
                continue
            expect.append(i)
        assert int(g[cell, 0]) == len(expect)
        assert sorted(int(g[cell, 2 + 2 * k]) for k in range(len(expect))) == expect


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n,seed", [(1, 64, 1), (3, 64, 5), (2, 128, 2), (3, 128, 9)])
def test_light_build_matches_oracle(vrt, orc, kind, n, seed):
    vox, _ = vrt.generate_scene(kind, n, seed)
    ctx = vrt.Context(0)
    sc = vrt.Scene(ctx, vox, n)
    st = sc.build_lights()
    words, alias, grid = sc.lights()
    ow, oweights = orc.light_list(vox, n)
    assert st.count == len(ow) > 0
    np.testing.assert_array_equal(words, ow)
    np.testing.assert_array_equal(alias, orc.light_alias(oweights))
    np.testing.assert_array_equal(grid, orc.light_grid(n, ow, oweights))
    assert st.total_weight == pytest.approx(float(np.sum(oweights)), rel=1e-12)
    # an edit that removes every emissive voxel in a box, then a rebuild
    sc.edit_box(0, 0, 0, n // 2 - 1, n - 1, n - 1, 0)
    st2 = sc.build_lights()
    v2, _, _ = sc.read()
    ow2, ow2w = orc.light_list(v2, n)
    w2, a2, g2 = sc.lights()
    assert st2.count == len(ow2)
    np.testing.assert_array_equal(w2, ow2)
    np.testing.assert_array_equal(a2, orc.light_alias(ow2w))
    np.testing.assert_array_equal(g2, orc.light_grid(n, ow2, ow2w))
