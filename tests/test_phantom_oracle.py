"""Phantom-builder oracle against the reference's own definitions:
SpinProperty's tables (src/phantom/SpinProperty.jl), generate_grid
(src/grid/Grid.jl:78-108), the fat shift of hophantom_brain
(src/phantom/hophantom_brain.jl:27-31), csm_Birdcage (src/phantom/csm/Birdcage.jl)
and the size invariants of test/unit/test_HOPhantom.jl:18-25."""
import numpy as np

from oracle import oracle as orc

CLASSES = [23, 46, 70, 93, 116, 139, 162, 185, 209, 232, 255]


def test_tissue_tables_at_1p5t_and_7t():
    lab = np.array(CLASSES + [0, 7], np.uint8)
    t1, t2, t2s, rho = orc.spin_property_np(lab, "1.5T")
    assert t1[1] == 833 * 1e-3 and t2[1] == 83 * 1e-3 and t2s[1] == 69 * 1e-3 and rho[1] == 0.86  # GM
    assert t1[0] == 2569 * 1e-3 and rho[5] == 0.7 and rho[6] == 0 and rho[7] == 0  # CSF, skin, skull, vessels
    assert np.all(t1[-2:] == 0) and np.all(rho[-2:] == 0)  # background and unknown classes
    t1, t2, t2s, rho7 = orc.spin_property_np(lab, "7T")
    assert t1[2] == 1200 * 1e-3 and t2[2] == 40 * 1e-3 and t2s[2] == 27 * 1e-3  # WM
    assert np.array_equal(rho7, rho)


def test_generate_grid_is_centred():
    g = orc.generate_grid_np([0.2, 0.02, 0.002], [4, 1, 3])
    assert g.shape == (4, 1, 3, 3)
    assert np.allclose(g[:, 0, 0, 0], [-0.075, -0.025, 0.025, 0.075], rtol=1e-15, atol=0)
    assert np.all(g[:, :, :, 1] == 0)
    assert np.allclose(g[0, 0, :, 2], [-0.002 / 3, 0, 0.002 / 3], rtol=1e-15)


def test_brain_phantom_sizes_mask_order_and_fat():
    rng = np.random.default_rng(0)
    lab = rng.choice(np.array(CLASSES + [0, 0, 1], np.uint8), size=(6, 5, 4))
    csm = rng.standard_normal((6, 5, 4, 3)) + 1j * rng.standard_normal((6, 5, 4, 3))
    p = orc.brain_phantom_np(lab, (2e-3, 2e-3, 3e-3), (1e-3, 0, -2e-3), csm=csm)
    ns = len(p["x"])
    keep = np.isin(lab, [23, 46, 70, 93, 116, 139, 209, 232, 255])
    assert ns == keep.sum() and p["csm"].shape == (ns, 3)
    # column-major order: the first kept voxel is the first in Fortran order
    first = np.flatnonzero(keep.ravel(order="F"))[0]
    ix, iy, iz = np.unravel_index(first, lab.shape, order="F")
    assert p["x"][0] == (ix - 2.5) * (6 * 2e-3 / 6) + 1e-3
    assert p["csm"][0, 2] == csm[ix, iy, iz, 2]
    fat = np.isin(lab.ravel(order="F")[keep.ravel(order="F")], [93, 209])
    assert np.all(p["dw"][fat] == -220 * (2 * np.pi)) and np.all(p["dw"][~fat] == 0)
    unit = orc.brain_phantom_np(lab, (2e-3, 2e-3, 3e-3))
    assert unit["csm"].shape == (ns, 1) and np.all(unit["csm"] == 1)


def test_birdcage_is_rss_normalised_and_rotates():
    m = orc.csm_birdcage_np(40, 30, 8, 1.5)
    assert m.shape == (40, 30, 8)
    assert np.allclose(np.sqrt(np.sum(np.abs(m) ** 2, axis=2)), 1.0, rtol=1e-14)
    # coil 0 sits at (+1.5, 0) in relative units: nearest to the x = nx-1 edge
    mag0 = np.abs(m[:, 15, 0])
    assert np.argmax(mag0) == 39
