"""Save points of a run: the static-cloud output record and the Lyman-alpha checkpoint.

The reference writes both to HDF5 (src/SaveHDF5Data_StaticCloudTests.jl:17-205, 329-425 and the
"Checkpoint" group of src/SaveHDF5Data_RHD_SingleStar.jl:161-175, 1315-1320). This image has
no HDF5 library, so the same datasets, under the same names and in the shapes an HDF5 reader in
C order sees, go to a NumPy .npz archive. Everything is computed on the device; a save point
downloads only what it stores (the edge-ring spectra and the step records between save points
stay on the device until then).
"""
import numpy as np


class StaticRunRecord:
    """The output file of a static-cloud run (CreateHDF5File / SaveHDF5Data of
    src/SaveHDF5Data_StaticCloudTests.jl): the grid once, then per save point the time, M_F and
    its radial-net/out parts, L, f_esc and the raw and normalised edge-ring spectra.

        rec = StaticRunRecord(cloud, n_saved)
        for s in range(n_saved):
            hist = ctx.static_steps(n_between, ...)       # step records stay on the device until here
            rec.save(ctx, s, t, hist[-1])
        rec.write("run.npz")
    """

    def __init__(self, cloud, n_saved):
        g = cloud.geom
        n_edge = None
        self.data = {"rCoM": np.asarray(g.rCoM), "ZCoM": np.asarray(g.ZCoM), "r": np.asarray(g.r),
                     "Z": np.asarray(g.Z), "CellVolumes": np.asarray(g.dV),
                     "Times": np.zeros(n_saved)}
        for k in ("M_F_History", "M_F_radial_net_History", "M_F_radial_out_History", "L_Lya_History",
                  "f_esc_Lya_History"):
            self.data[k] = np.zeros(n_saved)
        self.n_saved = n_saved
        self.n_nu = cloud.n_nu
        self._edge = n_edge

    def save(self, ctx, index, t, record):
        """Save point `index` at time t: `record` is the step record of that step (the
        lyd_diag row: M_F, radial-net, radial-out, L, f_esc, kmin, kmax)."""
        raw, norm, ri, zi = ctx.edge_spectra()
        if "J_Lya_EdgeSpectra" not in self.data:
            n = raw.shape[0]
            self.data["J_Lya_EdgeSpectra"] = np.zeros((self.n_saved, self.n_nu, n))
            self.data["J_Lya_EdgeSpectra_Norm"] = np.zeros((self.n_saved, self.n_nu, n))
            self.data["J_Lya_Edge_rIndex"] = ri + 1           # 1-based, as the reference stores them
            self.data["J_Lya_Edge_ZIndex"] = zi + 1
        d = self.data
        d["Times"][index] = t
        d["M_F_History"][index], d["M_F_radial_net_History"][index] = record[0], record[1]
        d["M_F_radial_out_History"][index], d["L_Lya_History"][index] = record[2], record[3]
        d["f_esc_Lya_History"][index] = record[4]
        d["J_Lya_EdgeSpectra"][index] = raw.T
        d["J_Lya_EdgeSpectra_Norm"][index] = norm.T

    def write(self, path):
        np.savez(path, **self.data)


def save_checkpoint(ctx, path, t_current=0.0, dt=0.0, step=0, e_lya=False):
    """The Lyman-alpha part of the reference's restart checkpoint: Checkpoint/J_Lya, H_r_Lya and
    H_Z_Lya (C-order shape (n_z, n_r, n_nu)), the attributes t_current, dt and step, and, with
    e_lya, the RHD sub-cycle's per-cell e_Lya."""
    d = {"Checkpoint/J_Lya": ctx.download("J"), "Checkpoint/H_r_Lya": ctx.download("H_r"),
         "Checkpoint/H_Z_Lya": ctx.download("H_Z"),
         "Checkpoint/attrs/t_current": np.float64(t_current), "Checkpoint/attrs/dt": np.float64(dt),
         "Checkpoint/attrs/step": np.int64(step)}
    if e_lya:
        d["Checkpoint/e_Lya"] = ctx.download("e_Lya")
    np.savez(path, **d)


def load_checkpoint(ctx, path):
    """Restart a context from save_checkpoint's archive: J, H and (as after AdvectLya!) the old
    J and H, and e_Lya when stored. Returns (t_current, dt, step)."""
    with np.load(path) as f:
        for name, key in (("J", "J_Lya"), ("H_r", "H_r_Lya"), ("H_Z", "H_Z_Lya")):
            a = f["Checkpoint/" + key]
            ctx.upload(name, a)
            ctx.upload(name + "_old", a)
        if "Checkpoint/e_Lya" in f.files:
            ctx.upload("e_Lya", f["Checkpoint/e_Lya"])
        return (float(f["Checkpoint/attrs/t_current"]), float(f["Checkpoint/attrs/dt"]),
                int(f["Checkpoint/attrs/step"]))
