"""Host resampling of the phantom's source volumes, on the CPU: the analytic
cases of the reference's test/unit/test_csm.jl:12-57 and
test_phantom_interfaces.jl:52-70, a linear off-resonance field, and (when the
reference's bundled receive map is present) its real-map border cases
(test_csm.jl:59-80)."""
import os

import numpy as np
import pytest

from homs.model import ArgumentError
from homs.phantom import resample_b0, resample_csm, resample_labels

# The reference's data files are read only when HOMS_REFERENCE_ROOT names its source tree.
REF = os.environ.get("HOMS_REFERENCE_ROOT", "")
_ref = (lambda *parts: os.path.join(REF, *parts)) if REF else (lambda *parts: "")
CSM_MAT = _ref("src", "phantom", "csm", "csm_4p0.mat")

SPACING = (0.004, 0.006, 0.008)
DIMS = (3, 4, 2)


def _field(x, y, z):
    return np.array([complex(2 + 100 * x - 20 * y + 30 * z, 0.5 - 80 * x + 60 * y + 25 * z),
                     complex(0.7 - 40 * x + 10 * y - 90 * z, 1.2 + 35 * x - 45 * y + 70 * z)])


def _axes():
    return [(np.arange(n) - (n - 1) / 2) * s for n, s in zip(DIMS, SPACING)]


def _source():
    ax = _axes()
    src = np.zeros(DIMS + (2,), np.complex128)
    for i in range(DIMS[0]):
        for j in range(DIMS[1]):
            for k in range(DIMS[2]):
                src[i, j, k] = _field(ax[0][i], ax[1][j], ax[2][k])
    return src


def _sample(point):
    return resample_csm(_source(), SPACING, (0.001, 0.001, 0.001), (1, 1, 1), point).reshape(-1)


def _unit(v):
    return v / np.sqrt(np.sum(np.abs(v) ** 2))


def test_linear_receive_field_is_exact():
    tol = 64 * np.finfo(float).eps
    for point in ((0.0, 0.0, 0.0), (0.0011, -0.0023, 0.0009)):
        assert np.allclose(_sample(point), _unit(_field(*point)), rtol=tol, atol=tol)


def test_receive_map_cells_and_faces():
    tol = 64 * np.finfo(float).eps
    ax = _axes()
    faces = [n * s / 2 for n, s in zip(DIMS, SPACING)]
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                point = (sx * faces[0], sy * faces[1], sz * faces[2])
                clamped = [min(max(p, a[0]), a[-1]) for p, a in zip(point, ax)]
                got = _sample(point)
                assert np.allclose(got, _unit(_field(*clamped)), rtol=tol, atol=tol)
                assert abs(np.sum(np.abs(got) ** 2) - 1) <= tol and np.all(np.isfinite(got))
    for axis in range(3):
        for sign in (-1, 1):
            point = [0.0, 0.0, 0.0]
            point[axis] = sign * np.nextafter(faces[axis], np.inf)
            assert np.all(_sample(tuple(point)) == 0)
    zeros = resample_csm(np.zeros(DIMS + (3,), np.complex128), SPACING, (0.002,) * 3, (5, 5, 5), (0.0, 0.0, 0.0))
    assert np.all(np.isfinite(zeros)) and np.all(zeros == 0)


def test_label_volume_on_its_own_grid_and_at_its_faces():
    data = np.arange(1, 25, dtype=np.uint8).reshape((2, 3, 4), order="F")
    spacing = (1e-3, 2e-3, 3e-3)
    assert np.array_equal(resample_labels(data, spacing, spacing, (2, 3, 4), (0.0, 0.0, 0.0)), data)
    for sign in (-1, 1):
        edge = resample_labels(data, spacing, spacing, (1, 1, 1), (sign * 1e-3, 0.0, 0.0))
        outside = resample_labels(data, spacing, spacing, (1, 1, 1), (sign * 1.1e-3, 0.0, 0.0))
        assert edge.item() != 0 and outside.item() == 0
    with pytest.raises(ArgumentError):
        resample_labels(data, (0.0, 1e-3, 1e-3), (1e-3,) * 3, (2, 3, 4), (0.0, 0.0, 0.0))
    with pytest.raises(ArgumentError):
        resample_labels(data, spacing, (1e-3,) * 3, (0, 3, 4), (0.0, 0.0, 0.0))


def test_label_volume_nearest_neighbour():
    rng = np.random.default_rng(4)
    data = rng.integers(0, 256, (20, 16, 12), dtype=np.uint8)
    out = resample_labels(data, (1e-3,) * 3, (2.5e-3, 2.5e-3, 3e-3), (8, 6, 4), (0.0007, -0.0011, 0.0004))
    # nearest source centre of each target centre, computed independently
    for i in range(8):
        for j in range(6):
            for k in range(4):
                t = ((i - 3.5) * 2.5e-3 + 0.0007, (j - 2.5) * 2.5e-3 - 0.0011, (k - 1.5) * 3e-3 + 0.0004)
                idx = [int(np.argmin(np.abs((np.arange(n) - (n - 1) / 2) * 1e-3 - c))) for n, c in
                       zip(data.shape, t)]
                assert out[i, j, k] == data[tuple(idx)]


def test_off_resonance_map_is_linear_inside_and_zero_outside():
    n = (9, 7, 5)
    res = (4e-3,) * 3
    ax = [(np.arange(m) - (m - 1) / 2) * r for m, r in zip(n, res)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    data = 3.0 + 1000 * X - 700 * Y + 250 * Z
    tgt_res, tgt_n, loc = (1.5e-3, 2e-3, 3e-3), (30, 20, 9), (0.001, -0.002, 0.0)
    out = resample_b0(data, res, tgt_res, tgt_n, loc)
    tx = [(np.arange(m) - (m - 1) / 2) * r + l for m, r, l in zip(tgt_n, tgt_res, loc)]
    TX, TY, TZ = np.meshgrid(*tx, indexing="ij")
    inside = (np.abs(TX) <= ax[0][-1]) & (np.abs(TY) <= ax[1][-1]) & (np.abs(TZ) <= ax[2][-1])
    want = np.where(inside, 3.0 + 1000 * TX - 700 * TY + 250 * TZ, 0.0)
    assert np.allclose(out, want, rtol=1e-12, atol=1e-12)
    assert inside.any() and (~inside).any()
    nan = data.copy()
    nan[:] = np.nan
    assert np.all(resample_b0(nan, res, tgt_res, tgt_n, loc) == 0)


@pytest.mark.skipif(not os.path.exists(CSM_MAT), reason="the reference's receive map is not present")
def test_real_receive_map_border():
    import scipy.io as sio
    src = sio.loadmat(CSM_MAT)["csm"]
    res = (4e-3,) * 3
    spacing = (1e-3,) * 3
    boundary = resample_csm(src, res, spacing, (1, 9, 6), (-0.0885, -0.0045, -0.017))
    centre = resample_csm(src, res, spacing, (1, 9, 6), (-0.088, -0.0045, -0.017))
    assert np.array_equal(boundary, centre) and np.all(np.isfinite(boundary))
    assert np.allclose(np.sum(np.abs(boundary) ** 2, axis=3), 1, rtol=1e-12)
    assert np.all(resample_csm(src, res, spacing, (1, 1, 1), (-0.0901, 0.0, 0.0)) == 0)
    face = resample_csm(src, res, spacing, (1, 1, 1), (-0.09, -0.0045, -0.017))
    beyond = resample_csm(src, res, spacing, (1, 1, 1), (-np.nextafter(0.09, 1), -0.0045, -0.017))
    assert abs(np.sum(np.abs(face) ** 2) - 1) <= 64 * np.finfo(float).eps
    assert np.all(beyond == 0)
    full = resample_csm(src, res, res, (2, 3, 1), (0.0, 0.0, 0.0))
    assert full.shape == (2, 3, 1, 32) and np.all(np.isfinite(full))


def test_generate_grid():
    """generate_grid (src/grid/Grid.jl:64-108) against the oracle's grid, and its argument checks."""
    from homs.phantom import generate_grid
    from oracle import oracle as orc
    for fov, n in (((0.2, 0.2, 0.07), (100, 100, 35)), ((0.1, 0.05, 0.004), (3, 4, 1))):
        assert np.array_equal(generate_grid(fov, n), orc.generate_grid_np(fov, n))
    with pytest.raises(ArgumentError):
        generate_grid((0.2, 0.2), (4, 4, 4))
    with pytest.raises(ArgumentError):
        generate_grid((0.2, 0.2, 0.2), (4, 4.5, 4))
    with pytest.raises(ArgumentError):
        generate_grid((0.2, -0.2, 0.2), (4, 4, 4))


BRAIN_MAT = _ref("src", "phantom", "brain3D_0.5_0.5_0.5.mat")
B0_MAT = _ref("src", "phantom", "b0map", "b0_4p0.mat")


@pytest.mark.skipif(not (os.path.exists(BRAIN_MAT) and os.path.exists(CSM_MAT) and os.path.exists(B0_MAT)),
                    reason="the reference's phantom volumes are not present")
def test_real_volumes_on_target_grids():
    """test_HOPhantom.jl: the brain phantom's volumes at 2 mm on the reference's
    2D and 3D target matrices and orientations (the device build itself is
    covered by the GPU tests on synthetic volumes)."""
    import scipy.io as sio
    from homs.phantom import generate_grid
    brain = sio.loadmat(BRAIN_MAT)["data"]
    csm = sio.loadmat(CSM_MAT)["csm"]
    b0 = sio.loadmat(B0_MAT)["b0"]
    res = (2e-3,) * 3
    for tm in ((100, 100, 10), (1, 100, 100), (100, 1, 100), (100, 100, 1), (10, 100, 100), (100, 10, 100)):
        lab = resample_labels(brain, (0.5e-3,) * 3, res, tm, (0.0, 0.0, 0.0))
        assert lab.shape == tm and lab.dtype == np.uint8 and (lab != 0).sum() > 0
        assert generate_grid(np.array(tm) * 2e-3, tm).shape == tm + (3,)
    tm = (100, 100, 10)
    cm = resample_csm(csm, (4e-3,) * 3, res, tm, (0.0, 0.0, 0.0))
    assert cm.shape == tm + (32,) and np.all(np.isfinite(cm))
    nz = np.abs(cm).sum(axis=3) > 0
    assert np.allclose(np.sum(np.abs(cm[nz]) ** 2, axis=1), 1, rtol=1e-12)
    fm = resample_b0(b0, (4e-3,) * 3, res, tm, (0.0, 0.0, 0.0))
    assert fm.shape == tm and np.all(np.isfinite(fm))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_voxel_centre_grid_geometry(dt):
    """test_grid.jl: generate_grid's centres and argument checks, and Grid's
    flattened coordinates against them."""
    from homs.phantom import Grid, generate_grid
    fov = np.array([0.2, 0.3, 0.004], dt)
    dims = [2, 3, 1]
    xyz = generate_grid(fov, dims)
    assert xyz.shape == (2, 3, 1, 3) and xyz.dtype == np.float64
    assert np.allclose(xyz[:, 0, 0, 0], np.array([-1, 1]) * float(fov[0]) / 4)
    assert np.allclose(xyz[0, :, 0, 1], np.array([-1, 0, 1]) * float(fov[1]) / 3)
    assert np.all(xyz[..., 2] == 0)
    spacing = (fov / np.array(dims)).astype(dt)
    g = Grid(*dims, *spacing)
    for axis, v in enumerate((g.x, g.y, g.z)):
        assert v.dtype == dt
        assert np.allclose(v, xyz[..., axis].ravel(order="F"), atol=np.finfo(dt).eps)
    with pytest.raises(ArgumentError):
        Grid(0, 3, 1, *spacing)
    with pytest.raises(ArgumentError):
        Grid(2, 3, 1, dt(0), spacing[1], spacing[2])
    with pytest.raises(ArgumentError):
        Grid(2, 3, 1, dt(np.inf), spacing[1], spacing[2])
    for bad_fov in ([0.0, 0.2, 0.2], [-1.0, 0.2, 0.2], [np.inf, 0.2, 0.2], [np.nan, 0.2, 0.2]):
        with pytest.raises(ArgumentError):
            generate_grid(bad_fov, [2, 3, 1])
    for bad_dims in ([0, 3, 1], [-1, 3, 1], [1.5, 3, 1], [np.inf, 3, 1], [np.nan, 3, 1]):
        with pytest.raises(ArgumentError):
            generate_grid([0.2, 0.3, 0.004], bad_dims)
    with pytest.raises(ArgumentError):
        generate_grid([0.2, 0.3], [2, 3, 1])
    assert repr(Grid(100, 100, 35, 0.002, 0.002, 0.002)) == \
        "Grid [ MatrixSize: 100 x 100 x 35, Resolution: 2.0 x 2.0 x 2.0 mm³ ]"
