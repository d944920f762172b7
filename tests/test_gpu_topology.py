"""hns_create_from_voxels: the device-built topology (the SOP's 26-neighbour padding dilation of
the active voxels and the leaf-dense grid over the leaves they touch, in NanoVDB order)
against a numpy restatement of the same set and the host NanoVDB sort, and the tables against
the host build (hns_create on the same leaves)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def leaves_of(points, padding):
    """Origins of the leaves that the box [p - padding, p + padding] (padding <= 8) of any point
    touches: the point's own leaf, and the neighbour leaf across a face on each axis where the box
    crosses it (local coordinate < padding: the -1 side; local + padding >= 8: the +1 side).
    Points are first reduced to distinct (leaf, crossing sides) pairs as packed integers."""
    p = np.asarray(points, dtype=np.int64).reshape(-1, 3)
    c, loc = p >> 3, p & 7
    lo, hi = loc < padding, loc + padding >= 8
    base = c.min(axis=0) - 1
    dims = c.max(axis=0) - base + 2
    cc = c - base
    side = sum((lo[:, d].astype(np.int64) << (2 * d)) | (hi[:, d].astype(np.int64) << (2 * d + 1)) for d in range(3))
    u = np.unique(((cc[:, 0] * dims[1] + cc[:, 1]) * dims[2] + cc[:, 2]) * 64 + side)
    bits, lin = u % 64, u // 64
    uc = np.stack([lin // (dims[1] * dims[2]), (lin // dims[2]) % dims[1], lin % dims[2]], axis=1)
    out = []
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                ok = np.ones(len(u), dtype=bool)
                for d, o in enumerate((dx, dy, dz)):
                    if o == -1:
                        ok &= (bits >> (2 * d)) & 1 == 1
                    elif o == 1:
                        ok &= (bits >> (2 * d + 1)) & 1 == 1
                q = uc[ok] + np.array([dx, dy, dz])
                out.append((q[:, 0] * dims[1] + q[:, 1]) * dims[2] + q[:, 2])
    lin = np.unique(np.concatenate(out))
    q = np.stack([lin // (dims[1] * dims[2]), (lin // dims[2]) % dims[1], lin % dims[2]], axis=1)
    return (q + base) * 8


def nanovdb_sorted(origins):
    from hnanosolver_b200 import lib as hl

    return hl.sort_leaves_nanovdb(np.asarray(origins, dtype=np.int32))


def _points(seed, n, spread, centre=(0, 0, 0)):
    rng = np.random.default_rng(seed)
    return (rng.integers(-spread, spread, size=(n, 3)) + np.asarray(centre)).astype(np.int32)


def test_dilation_matches_26_neighbour_morphology():
    """The numpy leaf set equals the leaves touched by a dense 3x3x3 binary dilation repeated
    `padding` times (OpenVDB's NN_FACE_EDGE_VERTEX voxel dilation), so it is the reference's set."""
    from scipy import ndimage

    rng = np.random.default_rng(3)
    pts = rng.integers(8, 56, size=(40, 3))
    for padding in (0, 1, 3, 8):
        dense = np.zeros((64, 64, 64), dtype=bool)
        dense[pts[:, 0], pts[:, 1], pts[:, 2]] = True
        if padding:
            dense = ndimage.binary_dilation(dense, structure=np.ones((3, 3, 3), dtype=bool), iterations=padding)
        on = np.argwhere(dense)
        ref = np.unique(on >> 3, axis=0) * 8
        assert np.array_equal(leaves_of(pts, padding), ref)


@pytest.mark.parametrize("padding", [0, 1, 3, 8])
@pytest.mark.parametrize("case", ["cluster", "across_root_tiles", "repeats"])
def test_leaves_and_order_match(dev, padding, case):
    from hnanosolver_b200 import lib as hl

    if case == "cluster":
        pts = _points(1, 20000, 60)
    elif case == "across_root_tiles":  # negative coordinates, and the x = 4096 and z = -4096 root-tile faces
        pts = np.concatenate([_points(2, 5000, 40, (4096, -10, 10)), _points(3, 5000, 40, (4000, 10, -4100))])
    else:
        pts = np.repeat(_points(4, 300, 20), 7, axis=0)
    g = hl.Grid(voxels=pts, padding=padding, voxel_size=0.1)
    got = g.leaf_origins()
    want = nanovdb_sorted(leaves_of(pts, padding))
    assert np.array_equal(got, want)
    assert g.is_nanovdb_order()
    g.close()


def test_device_input_equals_host_input(dev):
    from hnanosolver_b200 import lib as hl

    pts = _points(5, 50000, 100)
    a = hl.Grid(voxels=pts, padding=2, voxel_size=0.1)
    b = hl.Grid(voxels=torch.from_numpy(pts).to(dev).contiguous(), padding=2, voxel_size=0.1)
    assert np.array_equal(a.leaf_origins(), b.leaf_origins())
    a.close()
    b.close()


def test_tables_equal_host_build(dev):
    """Divergence and a red-black solve on the device-built grid equal those on the host-built
    grid with the same leaves, to the bit (same slots, neighbour table and leaf table)."""
    from hnanosolver_b200 import lib as hl

    pts = np.concatenate([_points(6, 30000, 50), _points(7, 3000, 20, (150, 0, 0))])
    gd = hl.Grid(voxels=pts, padding=3, voxel_size=0.1)
    gh = hl.Grid(gd.leaf_origins(), voxel_size=0.1)
    n = gd.num_voxels
    assert gh.num_voxels == n
    rng = np.random.default_rng(8)
    v = torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)).to(dev)
    outs = []
    for g in (gd, gh):
        div, p = torch.empty(n, device=dev), torch.empty(n, device=dev)
        torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
        g.divergence(v, div)
        g.rbgs(div, p, 20, 1.5, flags=hl.SOLVE_ZERO_INIT)
        torch.cuda.synchronize()
        outs.append((div.cpu(), p.cpu()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    gd.close()
    gh.close()


def test_rejects_bad_input(dev):
    from hnanosolver_b200 import lib as hl

    with pytest.raises(hl.HnsError):
        hl.Grid(voxels=_points(9, 10, 5), padding=9)
    with pytest.raises(hl.HnsError):
        hl.Grid(voxels=np.array([[1 << 23, 0, 0]], dtype=np.int32))


def test_shell_band_build_time(dev):
    """The shell workload's active voxels (a 32-voxel band around a radius-200 sphere, 15.1M
    voxels) with padding 2: the device build's time, printed, and its leaves equal the
    numpy set."""
    import time

    from hnanosolver_b200 import lib as hl

    c = np.arange(56, 456, dtype=np.int32)
    x, y = np.meshgrid(c, c, indexing="ij")
    pts = []
    for z in range(56, 456):
        r = np.sqrt((x - 256.0) ** 2 + (y - 256.0) ** 2 + (z - 256.0) ** 2)
        m = np.abs(r - 200.0) <= 16.0
        pts.append(np.stack([x[m], y[m], np.full(m.sum(), z, dtype=np.int32)], axis=1))
    pts = np.ascontiguousarray(np.concatenate(pts).astype(np.int32))
    dv = torch.from_numpy(pts).to(dev).contiguous()
    hl.Grid(voxels=dv, padding=2, voxel_size=0.1).close()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = hl.Grid(voxels=dv, padding=2, voxel_size=0.1)
    t = time.perf_counter() - t0
    print(f"shell band: {len(pts)} voxels -> {g.num_leaves} leaves in {t * 1e3:.1f} ms")
    assert np.array_equal(g.leaf_origins(), nanovdb_sorted(leaves_of(pts, 2)))
    g.close()
