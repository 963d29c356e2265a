/*
 * A C caller of libnrg_chem.so, written the way a Fortran host code binds
 * nrg_chem.h through ISO_C_BINDING: it builds a ghost-layered 3-D block of
 * column-major arrays cells(lb:ub, ...) for T, rho, each species' Y, Y_prod
 * and Y_prod2, E_f_prod and bc_markers, fills the interior from an input
 * file, steps it through nrg_chem_step and writes the interior outputs.
 *
 *   c_abi_driver MECH THERMO MOLAR IN OUT
 *
 * IN:  int32 nx, ny, nz, N; float64 dt; then, interior cells in Fortran order
 *      (i fastest): float64 T[n], rho[n], Y[N][n]; int8 bc[n].
 * OUT: float64 Y_prod[N][n], Y_prod2[N][n], E_f_prod[n]; int64 cells,
 *      cells_active, cells_bad, steps.
 *
 * Exit status: 0 ok; 2 usage or file error; 3 a call returned an error;
 * 4 a ghost cell was written; 5 the argument checks did not reject bad bounds.
 * Y_prod2 starts at 3.25 everywhere, so skipped cells must keep that value.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nrg_chem.h"

#define GHOST_MARK (-1.0)

static int fail(const char* what, nrg_chem* h, int rc) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, nrg_chem_last_error(h));
  return 3;
}

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s MECH THERMO MOLAR IN OUT\n", argv[0]);
    return 2;
  }
  FILE* in = fopen(argv[4], "rb");
  if (!in) return 2;
  int32_t hdr[4];
  double dt;
  if (fread(hdr, 4, 4, in) != 4 || fread(&dt, 8, 1, in) != 1) return 2;
  const int nx = hdr[0], ny = hdr[1], nz = hdr[2], N = hdr[3];
  if (nx < 1 || ny < 1 || nz < 1 || N < 1 || N > NRG_MAX_SPECIES) return 2;
  const long n = (long)nx * ny * nz;
  /* cells(0:nx+1, 0:ny+1, 0:nz+1): one ghost layer on every side */
  const long ex = nx + 2, ey = ny + 2, ez = nz + 2, total = ex * ey * ez;

  double* T = malloc(sizeof(double) * total);
  double* rho = malloc(sizeof(double) * total);
  double* Ef = malloc(sizeof(double) * total);
  signed char* bc = malloc((size_t)total);
  double *Y[NRG_MAX_SPECIES], *Yp[NRG_MAX_SPECIES], *Yp2[NRG_MAX_SPECIES];
  for (int k = 0; k < N; ++k) {
    Y[k] = malloc(sizeof(double) * total);
    Yp[k] = malloc(sizeof(double) * total);
    Yp2[k] = malloc(sizeof(double) * total);
  }
  for (long c = 0; c < total; ++c) {
    T[c] = 250.0; /* ghost cells: cold and marked, never read back */
    rho[c] = 1.0;
    Ef[c] = GHOST_MARK;
    bc[c] = 1;
    for (int k = 0; k < N; ++k) {
      Y[k][c] = 0.0;
      Yp[k][c] = GHOST_MARK;
      Yp2[k][c] = GHOST_MARK;
    }
  }
#define AT(i, j, k) ((((long)(k)) * ey + (j)) * ex + (i))
  double* buf = malloc(sizeof(double) * n);
  signed char* bbuf = malloc((size_t)n);
  int ok = 1;
  for (int a = 0; a < 2 + N && ok; ++a) {
    ok = fread(buf, 8, (size_t)n, in) == (size_t)n;
    double* dst = a == 0 ? T : a == 1 ? rho : Y[a - 2];
    long q = 0;
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) dst[AT(i, j, k)] = buf[q++];
  }
  ok = ok && fread(bbuf, 1, (size_t)n, in) == (size_t)n;
  fclose(in);
  if (!ok) return 2;
  {
    long q = 0;
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          bc[AT(i, j, k)] = bbuf[q++];
          for (int s = 0; s < N; ++s) Yp2[s][AT(i, j, k)] = 3.25;
        }
  }

  nrg_chem* h = NULL;
  int rc = nrg_chem_create(argv[1], argv[2], argv[3], 1.0, NRG_EACT_CAL_MOL, &h);
  if (rc != NRG_OK) return fail("nrg_chem_create", NULL, rc);
  int ns = 0, nr = 0;
  rc = nrg_chem_info(h, &ns, &nr);
  if (rc != NRG_OK || ns != N) return fail("nrg_chem_info", h, rc ? rc : -99);

  nrg_field_desc f;
  memset(&f, 0, sizeof(f));
  f.lb[0] = f.lb[1] = f.lb[2] = 0;
  f.ub[0] = nx + 1;
  f.ub[1] = ny + 1;
  f.ub[2] = nz + 1;
  f.lo[0] = f.lo[1] = f.lo[2] = 1;
  f.hi[0] = nx;
  f.hi[1] = ny;
  f.hi[2] = nz;
  f.T = T;
  f.p = NULL;
  f.rho = rho;
  for (int k = 0; k < N; ++k) {
    f.Y[k] = Y[k];
    f.Y_prod[k] = Yp[k];
    f.Y_prod2[k] = Yp2[k];
  }
  f.E_f_prod = Ef;
  f.bc_markers = bc;

  /* bounds that leave the array are an argument error, not a crash */
  nrg_field_desc bad = f;
  bad.hi[0] = nx + 2;
  if (nrg_chem_step(h, dt, &bad, NULL) != NRG_ERR_ARG) return 5;

  nrg_chem_stats st;
  rc = nrg_chem_step(h, dt, &f, &st);
  if (rc != NRG_OK) return fail("nrg_chem_step", h, rc);

  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx + 1; ++i) {
        const int ghost = i == 0 || j == 0 || k == 0 || i == nx + 1 || j == ny + 1 || k == nz + 1;
        if (!ghost) continue;
        const long c = AT(i, j, k);
        if (Ef[c] != GHOST_MARK) return 4;
        for (int s = 0; s < N; ++s)
          if (Yp[s][c] != GHOST_MARK || Yp2[s][c] != GHOST_MARK) return 4;
      }

  FILE* out = fopen(argv[5], "wb");
  if (!out) return 2;
  for (int a = 0; a < 2 * N + 1; ++a) {
    const double* src = a < N ? Yp[a] : a < 2 * N ? Yp2[a - N] : Ef;
    long q = 0;
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) buf[q++] = src[AT(i, j, k)];
    if (fwrite(buf, 8, (size_t)n, out) != (size_t)n) return 2;
  }
  const int64_t counts[4] = {st.cells, st.cells_active, st.cells_bad, st.steps};
  if (fwrite(counts, 8, 4, out) != 4) return 2;
  fclose(out);
  rc = nrg_chem_destroy(h);
  if (rc != NRG_OK) return 3;
  printf("stepped %ld cells (%lld active) through nrg_chem_step\n", n, (long long)st.cells_active);
  return 0;
}
