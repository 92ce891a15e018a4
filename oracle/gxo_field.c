/*
 * gxo_field.c -- ORACLE (test infrastructure only): the reference's CMS
 * field-map reader restated in C (ScalarCMSmagField::ReadVectorData,
 * GetFieldValueRZ, GetFieldValue, examples/magneticfield/simplifiedCMS/inc/
 * Geant/ScalarCMSmagField.h:162-331): 181 x 161 (r, z) lattice points, r outer,
 * dr = 50 mm to 9 m, dz = 200 mm over +-16 m; values read as float and stored
 * times 1 / (dr dz) in float; bilinear weights from the areas to the corners;
 * r and z clamped to the lattice; (Br, Bphi) rotated by the azimuth.
 */
#include "gxo.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define NR 181
#define NZ 161

float *gxo_field_map_load(const char *path)
{
  FILE *f = fopen(path, "r");
  if (!f) return NULL;
  float *m = (float *)calloc((size_t)NR * NZ * 4, sizeof(float));
  const float ainv = (float)(1.0 / (50.0f * 200.0f));
  char line[512];
  int ind = 0;
  while (fgets(line, sizeof(line), f)) {
    float r, phi, z, bz, br, bphi;
    if (sscanf(line, "R(mm)= %f phi(deg)= %f Z(mm)= %f Bz(tesla)= %f Br(tesla)= %f Bphi(tesla)= %f", &r, &phi, &z,
               &bz, &br, &bphi) != 6)
      continue;
    if (ind >= NR * NZ) break;
    m[4 * ind] = br * ainv;
    m[4 * ind + 1] = bphi * ainv;
    m[4 * ind + 2] = bz * ainv;
    ++ind;
  }
  fclose(f);
  if (ind != NR * NZ) {
    free(m);
    return NULL;
  }
  return m;
}

void gxo_field_map_free(float *map) { free(map); }

void gxo_field_map_value(const float *map, const double pos[3], double B[3])
{
  const float rdiff = 9000.0f / (NR - 1), zdiff = 2 * 16000.0f / (NZ - 1);
  const float rdinv = 1.0f / rdiff, zdinv = 1.0f / zdiff;
  double r0 = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double radius = fmin(r0, 9000.0), z = fmax(fmin(pos[2], 16000.0), -16000.0);
  double rfloor = floor(radius * rdinv), zind = floor((z - (-16000.0)) * zdinv);
  if (rfloor > NR - 2) rfloor = NR - 2;
  if (zind > NZ - 2) zind = NZ - 2;
  int i1 = (int)(rfloor * NZ + zind), i2 = i1 + 1;
  double zlow = (zind - (NZ - 1) / 2) * zdiff, zhigh = zlow + zdiff;
  double rlow = rfloor * rdiff, rhigh = rlow + rdiff;
  double a1 = (rhigh - radius) * (zhigh - z), a2 = (rhigh - radius) * (z - zlow);
  double a3 = (radius - rlow) * (zhigh - z), a4 = (radius - rlow) * (z - zlow);
  const float *b1 = map + 4 * i1, *b3 = map + 4 * (i1 + NZ), *b2 = map + 4 * i2, *b4 = map + 4 * (i2 + NZ);
  double br = b1[0] * a1 + b2[0] * a2 + b3[0] * a3 + b4[0] * a4;
  double bphi = b1[1] * a1 + b2[1] * a2 + b3[1] * a3 + b4[1] * a4;
  double bz = b1[2] * a1 + b2[2] * a2 + b3[2] * a3 + b4[2] * a4;
  double s = 0.0, c = 1.0;
  if (r0 != 0.0) {
    float rinv = (float)(1.0 / r0);
    s = pos[1] * rinv;
    c = pos[0] * rinv;
  }
  B[0] = br * c - bphi * s;
  B[1] = br * s + bphi * c;
  B[2] = bz;
}

void gxo_field_map_batch(const float *map, int n, const double *pos, double *B)
{
  for (int i = 0; i < n; ++i) gxo_field_map_value(map, pos + 3 * i, B + 3 * i);
}
