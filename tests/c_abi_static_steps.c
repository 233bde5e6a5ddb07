/* A plain C caller of the C ABI (include/lydion_m1.h): the calls a binding in another language
 * makes for the static-cloud driver, without Python in between.
 *
 *   c_abi_static_steps INPUT OUTPUT
 *
 * INPUT is a sequence of named records (a 32-byte NUL-padded name, an int64 count, then that
 * many doubles): "dims" (n_nu, n_r, n_z), "config" (flux method, recoil, kcore_min, kcore_max,
 * alpha_floor), the lyd_geometry arrays by field name ("dr_bnd" and "dZ_bnd" of 10), the
 * frequency grid ("nu", "nuC", "dnu", "inv_dnu", "inv_nuC"), uploads "up:<field id>", and "step"
 * (c_tilde, dt, z_center, bc_r_right, bc_z_bot, bc_z_top, n_steps). The program creates an FP64
 * context, sets geometry and frequency grid, uploads the fields, derives H_voigt and phi_nu on
 * the device, runs the steps and writes to OUTPUT the n_steps diagnostics records (7 doubles
 * each) and then the final J, H_r and H_Z. Exit status 0 on success. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lydion_m1.h"

typedef struct { char name[33]; int64_t n; double *v; } rec;

static rec *recs;
static int nrec;

static const rec *get(const char *name) {
    for (int q = 0; q < nrec; q++)
        if (strcmp(recs[q].name, name) == 0) return &recs[q];
    fprintf(stderr, "missing record %s\n", name);
    exit(2);
}

static int check(lyd_ctx *c, int rc, const char *what) {
    if (rc != LYD_OK) {
        fprintf(stderr, "%s: %d %s\n", what, rc, lyd_last_error(c));
        exit(3);
    }
    return rc;
}

int main(int argc, char **argv) {
    if (argc != 3) return 1;
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 1;
    int cap = 64;
    recs = (rec *)calloc(cap, sizeof(rec));
    char name[32];
    while (fread(name, 1, 32, f) == 32) {
        if (nrec == cap) recs = (rec *)realloc(recs, (cap *= 2) * sizeof(rec));
        rec *r = &recs[nrec++];
        memcpy(r->name, name, 32);
        r->name[32] = 0;
        if (fread(&r->n, sizeof(int64_t), 1, f) != 1) return 1;
        r->v = (double *)malloc((r->n > 0 ? r->n : 1) * sizeof(double));
        if ((int64_t)fread(r->v, sizeof(double), r->n, f) != r->n) return 1;
    }
    fclose(f);

    const double *dm = get("dims")->v, *cf = get("config")->v;
    lyd_dims dims = {0};
    dims.n_nu = (int32_t)dm[0]; dims.n_r = (int32_t)dm[1]; dims.n_z = (int32_t)dm[2];
    lyd_config cfg = {0};
    cfg.flux_method = (int32_t)cf[0]; cfg.recoil = (int32_t)cf[1]; cfg.precision = LYD_PREC_FP64;
    cfg.kcore_min = (int32_t)cf[2]; cfg.kcore_max = (int32_t)cf[3]; cfg.alpha_floor = cf[4];
    lyd_ctx *c = NULL;
    check(NULL, lyd_create(&c, &dims, &cfg), "lyd_create");

    lyd_geometry g;
    memset(&g, 0, sizeof(g));
    g.r = get("r")->v; g.Z = get("Z")->v; g.rCoM = get("rCoM")->v; g.ZCoM = get("ZCoM")->v;
    g.dV = get("dV")->v; g.inv_dV = get("inv_dV")->v; g.A_r = get("A_r")->v; g.A_Z = get("A_Z")->v;
    g.inv_r_cell = get("inv_r_cell")->v;
    g.dr_L = get("dr_L")->v; g.dr_R = get("dr_R")->v; g.inv_dr_i_im1 = get("inv_dr_i_im1")->v;
    g.inv_dr_ip1_i = get("inv_dr_ip1_i")->v; g.inv_dr_ip2_ip1 = get("inv_dr_ip2_ip1")->v;
    memcpy(g.dr_bnd, get("dr_bnd")->v, sizeof(g.dr_bnd));
    g.dZ_L = get("dZ_L")->v; g.dZ_R = get("dZ_R")->v; g.inv_dZ_j_jm1 = get("inv_dZ_j_jm1")->v;
    g.inv_dZ_jp1_j = get("inv_dZ_jp1_j")->v; g.inv_dZ_jp2_jp1 = get("inv_dZ_jp2_jp1")->v;
    memcpy(g.dZ_bnd, get("dZ_bnd")->v, sizeof(g.dZ_bnd));
    check(c, lyd_set_geometry(c, &g), "lyd_set_geometry");

    lyd_freq_grid fg;
    fg.nu = get("nu")->v; fg.nuC = get("nuC")->v; fg.dnu = get("dnu")->v;
    fg.inv_dnu = get("inv_dnu")->v; fg.inv_nuC = get("inv_nuC")->v;
    check(c, lyd_set_freq_grid(c, &fg), "lyd_set_freq_grid");

    for (int q = 0; q < nrec; q++)
        if (strncmp(recs[q].name, "up:", 3) == 0)
            check(c, lyd_upload(c, atoi(recs[q].name + 3), recs[q].v, (size_t)recs[q].n), recs[q].name);
    check(c, lyd_update_hvoigt(c), "lyd_update_hvoigt");
    check(c, lyd_update_phi_nu(c, cfg.kcore_min, cfg.kcore_max), "lyd_update_phi_nu");

    const double *sp = get("step")->v;
    lyd_step_params p;
    memset(&p, 0, sizeof(p));
    p.c_tilde = sp[0]; p.dt = sp[1]; p.z_center = sp[2];
    p.bc_r_right = (int32_t)sp[3]; p.bc_z_bot = (int32_t)sp[4]; p.bc_z_top = (int32_t)sp[5];
    p.n_steps = (int32_t)sp[6];
    lyd_diag *hist = (lyd_diag *)calloc(p.n_steps, sizeof(lyd_diag));
    check(c, lyd_static_steps(c, &p, hist), "lyd_static_steps");

    const size_t n3 = (size_t)dims.n_nu * dims.n_r * dims.n_z;
    double *state = (double *)malloc(3 * n3 * sizeof(double));
    check(c, lyd_download(c, LYD_F_J, state, n3), "lyd_download J");
    check(c, lyd_download(c, LYD_F_H_R, state + n3, n3), "lyd_download H_r");
    check(c, lyd_download(c, LYD_F_H_Z, state + 2 * n3, n3), "lyd_download H_Z");
    FILE *o = fopen(argv[2], "wb");
    if (!o) return 1;
    for (int s = 0; s < p.n_steps; s++) {
        const double d[7] = {hist[s].M_F, hist[s].M_F_radial_net, hist[s].M_F_radial_out, hist[s].L_tot,
                             hist[s].f_esc, (double)hist[s].kmin, (double)hist[s].kmax};
        fwrite(d, sizeof(double), 7, o);
    }
    fwrite(state, sizeof(double), 3 * n3, o);
    fclose(o);
    check(c, lyd_destroy(c), "lyd_destroy");
    return 0;
}
