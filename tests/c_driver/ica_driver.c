/*
 * A plain-C stand-in for the reference's three kernel drivers
 * (kernels/NICAM/{dyn_horiz_adv_flux,dyn_horiz_adv_limiter,dyn_vert_adv_limiter}/src/main.f90):
 * one process's arrays of one region with both poles, sized by the drivers' module globals
 * (problem_size.inc:28-50: ADM_lall = 1, ADM_have_pl = .true., ADM_have_sgp(1) = .true.),
 * handed to the library's C ABI exactly as a Fortran driver would hand them over through the
 * ISO_C_BINDING shim: ica_init_regions, ica_set_geometry, then ica_horizontal_flux,
 * ica_horizontal_limiter_thuburn (Qout_post given, as the drivers read it from their
 * snapshot) and ica_vertical_limiter_thuburn on host arrays.
 *
 *   ica_driver <dir> <gall_1d> <kall> <dt>
 *
 * Inputs are <dir>/<name>.f64 (native-endian doubles in the library's C layout, Fortran
 * var(ij,k,l,m) = C [m][l][k][ij]); outputs go to <dir>/out_<name>.f64.  The output arrays
 * start from the input files of the same name (flx_h, q_a, q_h ...), as the drivers' do.
 * Exit status 0 on success; a library error prints ica_last_error() and exits 1.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "icoadv.h"

static const char *g_dir;

static double *load(const char *name, size_t n) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s.f64", g_dir, name);
  FILE *f = fopen(path, "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  double *a = malloc(n * sizeof(double));
  if (!a || fread(a, sizeof(double), n, f) != n) { fprintf(stderr, "short read %s\n", path); exit(2); }
  fclose(f);
  return a;
}

static void save(const char *name, const double *a, size_t n) {
  char path[4096];
  snprintf(path, sizeof path, "%s/out_%s.f64", g_dir, name);
  FILE *f = fopen(path, "wb");
  if (!f || fwrite(a, sizeof(double), n, f) != n) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
  fclose(f);
}

#define CHECK(call)                                                        \
  do {                                                                     \
    int rc_ = (call);                                                      \
    if (rc_ != ICA_OK) {                                                   \
      fprintf(stderr, "%s: %d: %s\n", #call, rc_, ica_last_error());       \
      return 1;                                                            \
    }                                                                      \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s <dir> <gall_1d> <kall> <dt>\n", argv[0]);
    return 2;
  }
  g_dir = argv[1];
  const int gall_1d = atoi(argv[2]), kall = atoi(argv[3]);
  const double dt = atof(argv[4]);
  const int lall = 1, have_pl = 1, have_sgp[1] = {1};
  const size_t G = (size_t)gall_1d * gall_1d, K = (size_t)kall, L = lall, P = 6 * K * 2;

  ica_ctx *ctx = NULL;
  CHECK(ica_init_regions(gall_1d, kall, 2, kall - 1, lall, have_pl, have_sgp, 0, &ctx));
  ica_sizes sz;
  CHECK(ica_get_sizes(ctx, &sz));
  if (sz.gall != (int)G || sz.lall != lall || sz.kmin != 2 || sz.kmax != kall - 1) {
    fprintf(stderr, "unexpected sizes\n");
    return 1;
  }

  /* metrics of mod_misc (no K0 axis in the library's layout) */
  double *GRD_xr = load("GRD_xr", 9 * G * L), *GRD_xr_pl = load("GRD_xr_pl", 3 * 12);
  double *GMTR_p = load("GMTR_p", 8 * G * L), *GMTR_p_pl = load("GMTR_p_pl", 8 * 12);
  double *GMTR_t = load("GMTR_t", 10 * G * L), *GMTR_t_pl = load("GMTR_t_pl", 5 * 12);
  double *GMTR_a = load("GMTR_a", 36 * G * L), *GMTR_a_pl = load("GMTR_a_pl", 18 * 12);
  CHECK(ica_set_geometry(ctx, GRD_xr, GRD_xr_pl, GMTR_p, GMTR_p_pl, GMTR_t, GMTR_t_pl, GMTR_a, GMTR_a_pl));

  /* dyn_horiz_adv_flux/src/main.f90:229-235 */
  double *flx_h = load("flx_h", 6 * G * K * L), *flx_h_pl = load("flx_h_pl", P);
  double *GRD_xc = load("GRD_xc", 9 * G * K * L), *GRD_xc_pl = load("GRD_xc_pl", 3 * P);
  double *rho = load("rho", G * K * L), *rho_pl = load("rho_pl", P);
  double *vx = load("rhovx", G * K * L), *vx_pl = load("rhovx_pl", P);
  double *vy = load("rhovy", G * K * L), *vy_pl = load("rhovy_pl", P);
  double *vz = load("rhovz", G * K * L), *vz_pl = load("rhovz_pl", P);
  CHECK(ica_horizontal_flux(ctx, flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl,
                            dt));
  save("flx_h", flx_h, 6 * G * K * L);
  save("flx_h_pl", flx_h_pl, P);
  save("GRD_xc", GRD_xc, 9 * G * K * L);
  save("GRD_xc_pl", GRD_xc_pl, 3 * P);

  /* dyn_horiz_adv_limiter/src/main.f90: the limiter with the snapshot's Qout_post */
  double *q_a = load("q_a", 6 * G * K * L), *q_a_pl = load("q_a_pl", P);
  double *q = load("q", G * K * L), *q_pl = load("q_pl", P);
  double *d = load("d", G * K * L), *d_pl = load("d_pl", P);
  double *ch = load("ch", 6 * G * K * L), *ch_pl = load("ch_pl", P);
  double *cm = load("cmask", 6 * G * K * L), *cm_pl = load("cmask_pl", P);
  double *qo = calloc(2 * G * K * L, sizeof(double)), *qo_pl = calloc(2 * P, sizeof(double));
  double *post = load("Qout_post", 2 * G * K * L), *post_pl = load("Qout_post_pl", 2 * P);
  CHECK(ica_horizontal_limiter_thuburn(ctx, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cm, cm_pl, qo, qo_pl, post,
                                       post_pl));
  save("q_a", q_a, 6 * G * K * L);
  save("q_a_pl", q_a_pl, P);
  save("Qout_prev", qo, 2 * G * K * L);
  save("Qout_prev_pl", qo_pl, 2 * P);
  /* a context without a region topology has no halo fill: the on-GPU Qout fill is refused */
  if (ica_horizontal_limiter_thuburn(ctx, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cm, cm_pl, qo, qo_pl, NULL,
                                     NULL) != ICA_ERR_STATE ||
      ica_comm_data_transfer(ctx, q, q_pl, kall, 1) != ICA_ERR_STATE) {
    fprintf(stderr, "a partial-grid context accepted a halo fill\n");
    return 1;
  }

  /* dyn_vert_adv_limiter/src/main.f90 */
  double *q_h = load("q_h", G * K * L), *q_h_pl = load("q_h_pl", P);
  double *vq = load("vq", G * K * L), *vq_pl = load("vq_pl", P);
  double *vd = load("vd", G * K * L), *vd_pl = load("vd_pl", P);
  double *ck = load("ck", 2 * G * K * L), *ck_pl = load("ck_pl", 2 * P);
  CHECK(ica_vertical_limiter_thuburn(ctx, q_h, q_h_pl, vq, vq_pl, vd, vd_pl, ck, ck_pl));
  save("q_h", q_h, G * K * L);
  save("q_h_pl", q_h_pl, P);

  const long long launches = ica_launch_count(ctx);
  CHECK(ica_finalize(ctx));
  printf("ica_driver ok: gall_1d %d, kall %d, lall %d, %lld kernels\n", gall_1d, kall, lall, launches);
  return 0;
}
