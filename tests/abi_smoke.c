/* The C ABI from C (and, compiled as C++, from C++): links against
 * libem2g.so through include/em2g.h only.
 *
 *   abi_smoke cpu   parameter validation, no device call
 *   abi_smoke gpu   a uniform plasma in zero fields: one em2g_step, then
 *                   charge conservation of the deposit (sum of rho over the
 *                   cells = total macro charge), ake > 0, particles returned
 *                   in slot order with positions moved by v dt
 * Prints "ok" and exits 0 on success. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "em2g.h"

#define CHECK(cond, msg)                                                    \
  do {                                                                      \
    if (!(cond)) {                                                          \
      fprintf(stderr, "FAIL %s: %s (%s)\n", msg, #cond, em2g_last_error()); \
      return 1;                                                             \
    }                                                                       \
  } while (0)

static int cpu_checks(void) {
  em2g_params p;
  em2g_ctx *c = NULL;
  CHECK(em2g_abi_version() == EM2G_ABI_VERSION, "abi version");
  CHECK(em2g_params_init(&p) == EM2G_OK, "params_init");
  CHECK(p.struct_size == sizeof(em2g_params), "struct size");
  p.nx = 2;
  p.ny = 16;
  CHECK(em2g_create(&p, &c) == EM2G_ERR_INVALID && c == NULL, "nx < 4 rejected");
  CHECK(strstr(em2g_last_error(), "nx") != NULL, "message names nx");
  CHECK(em2g_params_init(NULL) == EM2G_ERR_INVALID, "null params");
  CHECK(em2g_destroy(NULL) == EM2G_OK, "destroy(NULL)");
  return 0;
}

static int gpu_checks(void) {
  const int nx = 32, ny = 16, npc = 4;
  const int64_t n = (int64_t)nx * ny * npc;
  const int64_t w = (int64_t)(nx + 3) * (ny + 3);
  em2g_params p;
  em2g_ctx *c = NULL;
  em2g_params_init(&p);
  p.nx = nx;
  p.ny = ny;
  p.nsp = 1;
  p.dx = p.dy = 0.5;
  p.dt = 0.05;
  p.qm[0] = -1.0;
  p.q[0] = -0.01;
  p.dn[0] = 1.0;
  p.am[0] = 0.01;
  p.np_max[0] = n;
  CHECK(em2g_create(&p, &c) == EM2G_OK, "create");
  double *buf = (double *)calloc((size_t)(6 * n + 13 * w), sizeof(double));
  double *x = buf, *y = x + n, *vx = y + n, *vy = vx + n, *vz = vy + n, *g = vz + n;
  double *fld = g + n;
  srand(7);
  for (int64_t j = 0; j < n; ++j) {
    x[j] = nx * (rand() / (RAND_MAX + 1.0));
    y[j] = ny * (rand() / (RAND_MAX + 1.0));
    vx[j] = 0.2 * (rand() / (RAND_MAX + 1.0) - 0.5);
    vy[j] = 0.2 * (rand() / (RAND_MAX + 1.0) - 0.5);
    vz[j] = 0.0;
    g[j] = 1.0 / sqrt(1.0 - vx[j] * vx[j] - vy[j] * vy[j]);
  }
  CHECK(em2g_set_fields(c, fld) == EM2G_OK, "set_fields");
  CHECK(em2g_set_particles(c, 0, n, x, y, vx, vy, vz, g) == EM2G_OK, "set_particles");
  double ake[4] = {0, 0, 0, 0};
  CHECK(em2g_move(c, ake) == EM2G_OK && ake[0] > 0.0, "move / ake");
  CHECK(em2g_curnt(c) == EM2G_OK, "curnt");
  /* rho after curnt, before fields folds it: all charge is in the array */
  CHECK(em2g_get_field(c, EM2G_RHO, fld) == EM2G_OK, "get rho");
  double q = 0.0;
  for (int64_t k = 0; k < w; ++k) q += fld[k];
  const double want = n * p.q[0] * p.dn[0] / (p.dx * p.dy);
  CHECK(fabs(q - want) < 1e-9 * fabs(want), "charge conservation of the deposit");
  int iters = -1;
  CHECK(em2g_fields(c, 1, NULL, &iters) == EM2G_OK && iters >= 1, "fields");
  double *x2 = (double *)malloc(sizeof(double) * 6 * n);
  int64_t m = 0;
  CHECK(em2g_get_particles(c, 0, &m, x2, x2 + n, x2 + 2 * n, x2 + 3 * n, x2 + 4 * n,
                           x2 + 5 * n) == EM2G_OK && m == n, "get_particles");
  for (int64_t j = 0; j < n; ++j) {
    double dxp = x2[j] - x[j];
    if (dxp > nx / 2) dxp -= nx;
    if (dxp < -nx / 2) dxp += nx;
    /* zero fields: v unchanged, x moved by v dt / dx (pic/curnt.f90:181) */
    CHECK(fabs(dxp - vx[j] * p.dt / p.dx) < 1e-12, "particle moved by v dt");
  }
  CHECK(em2g_destroy(c) == EM2G_OK, "destroy");
  free(x2);
  free(buf);
  return 0;
}

int main(int argc, char **argv) {
  int rc = cpu_checks();
  if (!rc && argc > 1 && strcmp(argv[1], "gpu") == 0) rc = gpu_checks();
  if (!rc) printf("ok\n");
  return rc;
}
