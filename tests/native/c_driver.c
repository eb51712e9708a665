/* A plain C99 host of the solver, as a C or Fortran caller links it: reads a
 * 1D problem from a raw little-endian file, calls evp1d_init / evp1d_run /
 * evp1d_finalize with host pointers (the dyn_evp1d_init / dyn_evp1d_run /
 * dyn_evp1d_finalize sequence, integration/ice_dyn_evp1d.F90:65-331) and
 * writes the results.  Test code only.
 *
 * Input:  int32 na, navel, ndte; int32 ee, ne, se, nw, sw, sse, skipT,
 *         skipU [na]; float64 dxT, dyT, HTE, HTN, HTEm1, HTNm1, uarear [na];
 *         the 12 stresses [na]; strength, Cw, aiu, uocn, vocn, waterx, watery,
 *         forcex, forcey, umassdti, fm, Tbu [na]; uvel, vvel [navel];
 *         strintx, strinty, Cb [na].
 * Output: the 12 stresses [na], uvel, vvel [navel], strintx, strinty, Cb [na]. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "evp1d.h"

static FILE *in;

static void *take(size_t n, size_t size) {
  void *p = malloc(n * size + 1);
  if (!p || fread(p, size, n, in) != n) {
    fprintf(stderr, "short input\n");
    exit(3);
  }
  return p;
}

static void put(FILE *f, const double *a, size_t n) {
  if (fwrite(a, sizeof(double), n, f) != n) exit(4);
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  in = fopen(argv[1], "rb");
  if (!in) return 2;
  int32_t hdr[3];
  if (fread(hdr, sizeof(int32_t), 3, in) != 3) return 3;
  const int na = hdr[0], navel = hdr[1], ndte = hdr[2];
  int32_t *nb[6], *skip[2];
  double *geo[7], *stress[12], *f[12];
  for (int k = 0; k < 6; k++) nb[k] = take((size_t)na, sizeof(int32_t));
  for (int k = 0; k < 2; k++) skip[k] = take((size_t)na, sizeof(int32_t));
  for (int k = 0; k < 7; k++) geo[k] = take((size_t)na, sizeof(double));
  for (int k = 0; k < 12; k++) stress[k] = take((size_t)na, sizeof(double));
  for (int k = 0; k < 12; k++) f[k] = take((size_t)na, sizeof(double));
  double *uvel = take((size_t)navel, sizeof(double)), *vvel = take((size_t)navel, sizeof(double));
  double *strintx = take((size_t)na, sizeof(double)), *strinty = take((size_t)na, sizeof(double));
  double *Cb = take((size_t)na, sizeof(double));
  fclose(in);

  evp1d_params p;
  evp1d_set_evp_parameters(&p, ndte);
  evp1d_t *h = NULL;
  int rc = evp1d_init(&h, na, navel, nb[0], nb[1], nb[2], nb[3], nb[4], nb[5], geo[0], geo[1],
                      geo[2], geo[3], geo[4], geo[5], geo[6], &p, 0);
  if (rc != EVP1D_OK) {
    fprintf(stderr, "evp1d_init: %d %s\n", rc, evp1d_last_error());
    return 1;
  }
  evp1d_fields io;
  memset(&io, 0, sizeof io);
  io.skipT = skip[0];
  io.skipU = skip[1];
  for (int k = 0; k < 12; k++) io.stress[k] = stress[k];
  io.strength = f[0];
  io.Cw = f[1];
  io.aiu = f[2];
  io.uocn = f[3];
  io.vocn = f[4];
  io.waterx = f[5];
  io.watery = f[6];
  io.forcex = f[7];
  io.forcey = f[8];
  io.umassdti = f[9];
  io.fm = f[10];
  io.Tbu = f[11];
  io.uvel = uvel;
  io.vvel = vvel;
  io.strintx = strintx;
  io.strinty = strinty;
  io.Cb = Cb;
  rc = evp1d_run(h, ndte, &io);
  if (rc != EVP1D_OK) {
    fprintf(stderr, "evp1d_run: %d %s\n", rc, evp1d_last_error());
    evp1d_finalize(h);
    return 1;
  }
  rc = evp1d_finalize(h);
  if (rc != EVP1D_OK) return 1;

  FILE *out = fopen(argv[2], "wb");
  if (!out) return 2;
  for (int k = 0; k < 12; k++) put(out, stress[k], (size_t)na);
  put(out, uvel, (size_t)navel);
  put(out, vvel, (size_t)navel);
  put(out, strintx, (size_t)na);
  put(out, strinty, (size_t)na);
  put(out, Cb, (size_t)na);
  fclose(out);
  printf("ok %d %d %d\n", na, navel, ndte);
  return 0;
}
