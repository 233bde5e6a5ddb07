"""Host-side layouts without a GPU: the Z-slab partition of one field and the static-run record's
datasets (the names and shapes of src/SaveHDF5Data_StaticCloudTests.jl)."""
import numpy as np
import pytest

from lydion_b200 import domain as D
from lydion_b200 import snapshots
from lydion_b200 import workloads as W


@pytest.mark.parametrize("nz,n", [(9, 2), (256, 3), (64, 8), (17, 4)])
def test_slab_partition_covers_the_rows(nz, n):
    parts = D.slab_partition(nz, n)
    assert parts[0][0] == 0 and parts[-1][1] == nz
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))          # contiguous, no overlap
    sizes = [b - a for a, b in parts]
    assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 2
    for r in range(n):
        j0, j1, hb, ht = D.slab_layout(nz, n, r)
        assert (j0, j1) == parts[r]
        assert hb == (0 if r == 0 else 2) and ht == (0 if r == n - 1 else 2)


def test_slab_partition_rejects_thin_slabs():
    with pytest.raises(ValueError):
        D.slab_partition(7, 4)


def test_local_cloud_slices_rows_and_faces():
    cl = W.small_cloud()
    j0, j1, hb, ht = D.slab_layout(cl.nz, 2, 1)
    loc = D.local_cloud(cl, j0, j1, hb, ht)
    a, b = j0 - hb, j1 + ht
    assert loc.geom.ZCoM.shape[0] == b - a and loc.geom.A_Z.shape[0] == b - a + 1
    np.testing.assert_array_equal(loc.alpha, cl.alpha[a:b])
    np.testing.assert_array_equal(loc.u_Z_star, cl.u_Z_star[a:b + 1])
    np.testing.assert_array_equal(loc.geom.rCoM, cl.geom.rCoM)          # r is not split


class _FakeCtx:
    """edge_spectra() of a context: raw and normalised [edge, bin] with 0-based cell indices."""

    def __init__(self, n_edge, n_nu, seed):
        rng = np.random.default_rng(seed)
        self.raw = rng.random((n_edge, n_nu))
        self.norm = self.raw / self.raw.sum(1, keepdims=True)
        self.ri = np.arange(n_edge) % 5
        self.zi = np.arange(n_edge) // 5

    def edge_spectra(self):
        return self.raw, self.norm, self.ri, self.zi


def test_static_run_record_datasets(tmp_path):
    cl = W.small_cloud()
    rec = snapshots.StaticRunRecord(cl, 3)
    ctxs = [_FakeCtx(7, cl.n_nu, s) for s in range(3)]
    for s, ctx in enumerate(ctxs):
        rec.save(ctx, s, 0.5 * s, [1.0 + s, 2.0, 3.0, 4.0, 0.1 * s, 0, cl.n_nu - 1])
    path = str(tmp_path / "run.npz")
    rec.write(path)
    d = np.load(path)
    for k in ("rCoM", "ZCoM", "r", "Z", "CellVolumes", "Times", "M_F_History", "M_F_radial_net_History",
              "M_F_radial_out_History", "L_Lya_History", "f_esc_Lya_History", "J_Lya_EdgeSpectra",
              "J_Lya_EdgeSpectra_Norm", "J_Lya_Edge_rIndex", "J_Lya_Edge_ZIndex"):
        assert k in d, k
    assert d["J_Lya_EdgeSpectra"].shape == (3, cl.n_nu, 7)           # [save, bin, edge]
    np.testing.assert_array_equal(d["J_Lya_EdgeSpectra"][2], ctxs[2].raw.T)
    np.testing.assert_array_equal(d["J_Lya_Edge_rIndex"], ctxs[0].ri + 1)   # 1-based, as stored
    np.testing.assert_array_equal(d["Times"], [0.0, 0.5, 1.0])
    np.testing.assert_array_equal(d["M_F_History"], [1.0, 2.0, 3.0])
