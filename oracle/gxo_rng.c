/*
 * gxo_rng.c -- ORACLE (test infrastructure only): MRG32k3a restated from
 * source/Geant/random/MRG.hpp and source/Geant/random/src/MRG32k3a.cpp of the
 * reference (L'Ecuyer's RngStream combined multiple recursive generator).
 */
#include "gxo.h"

#include <math.h>
#include <string.h>

/* source/Geant/random/MRG.hpp:39-48 (published MRG32k3a parameters) */
static const double m1 = 4294967087.0;
static const double m2 = 4294944443.0;
static const double norm = 1.0 / (4294967087.0 + 1.0);
static const double a12 = 1403580.0;
static const double a13n = 810728.0;
static const double a21 = 527612.0;
static const double a23n = 1370589.0;
static const double two17 = 131072.0;
static const double two53 = 9007199254740992.0;

/* MRG.hpp:52-80: transition matrices, their 2^127 powers and inverses */
static const double A1p127[3][3] = {{2427906178.0, 3580155704.0, 949770784.0},
                                    {226153695.0, 1230515664.0, 3580155704.0},
                                    {1988835001.0, 986791581.0, 1230515664.0}};
static const double A2p127[3][3] = {{1464411153.0, 277697599.0, 1610723613.0},
                                    {32183930.0, 1464411153.0, 1022607788.0},
                                    {2824425944.0, 32183930.0, 2093834863.0}};
static const double A1p76[3][3] = {{82758667.0, 1871391091.0, 4127413238.0},
                                   {3672831523.0, 69195019.0, 1871391091.0},
                                   {3672091415.0, 3528743235.0, 69195019.0}};
static const double A2p76[3][3] = {{1511326704.0, 3759209742.0, 1610795712.0},
                                   {4292754251.0, 1511326704.0, 3889917532.0},
                                   {3859662829.0, 4292754251.0, 3708466080.0}};
static const double A1p0[3][3] = {{0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}, {-810728.0, 1403580.0, 0.0}};
static const double A2p0[3][3] = {{0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}, {-1370589.0, 0.0, 527612.0}};
static const double InvA1[3][3] = {{184888585.0, 0.0, 1945170933.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}};
static const double InvA2[3][3] = {{0.0, 360363334.0, 4225571728.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}};

/* One step of the two component recurrences, MRG32k3a::Kernel host branch,
 * MRG32k3a.cpp:124-163; returns the draw numerator z in [1, m1]. */
static double mrg_step(double *s)
{
  double k, p1, p2;
  p1 = a12 * s[1] - a13n * s[0];
  k = floor(p1 / m1);
  p1 -= k * m1;
  if (p1 < 0.) p1 += m1;
  s[0] = s[1];
  s[1] = s[2];
  s[2] = p1;
  p2 = a21 * s[5] - a23n * s[3];
  k = floor(p2 / m2);
  p2 -= k * m2;
  if (p2 < 0.) p2 += m2;
  s[3] = s[4];
  s[4] = s[5];
  s[5] = p2;
  return (p1 > p2) ? (p1 - p2) : (p1 - p2 + m1);
}

/* MRG32k3a::Kernel: u = z * norm, MRG32k3a.cpp:157 */
double gxo_mrg_u01(gxo_mrg_t *r) { return mrg_step(r->s) * norm; }

/* The integer numerator z (1 <= z <= m1) of one draw, u = z / (m1 + 1). */
uint32_t gxo_mrg_next_raw(gxo_mrg_t *r) { return (uint32_t)mrg_step(r->s); }

/* MultModM, MRG32k3a.cpp:207-230: (a*s + c) mod m with a, s, c, m < 2^35 */
static double mult_mod_m(double a, double s, double c, double m)
{
  double v;
  long a1;
  v = a * s + c;
  if (v >= two53 || v <= -two53) {
    a1 = (long)(a / two17);
    a -= a1 * two17;
    v = a1 * s;
    a1 = (long)(v / m);
    v -= a1 * m;
    v = v * two17 + a * s + c;
  }
  a1 = (long)(v / m);
  if ((v -= a1 * m) < 0.0) return v += m;
  return v;
}

/* MatVecModM, MRG32k3a.cpp:232-248 */
static void mat_vec_mod_m(const double A[3][3], const double s[3], double v[3], double m)
{
  double x[3];
  for (int i = 0; i < 3; ++i) {
    x[i] = mult_mod_m(A[i][0], s[0], 0.0, m);
    x[i] = mult_mod_m(A[i][1], s[1], x[i], m);
    x[i] = mult_mod_m(A[i][2], s[2], x[i], m);
  }
  for (int i = 0; i < 3; ++i) v[i] = x[i];
}

/* MatMatModM, MRG32k3a.cpp:250-269 */
static void mat_mat_mod_m(const double A[3][3], const double B[3][3], double C[3][3], double m)
{
  double V[3], W[3][3];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) V[j] = B[j][i];
    mat_vec_mod_m(A, V, V, m);
    for (int j = 0; j < 3; ++j) W[j][i] = V[j];
  }
  memcpy(C, W, sizeof(W));
}

/* MatTwoPowModM, MRG32k3a.cpp:271-287 */
static void mat_two_pow_mod_m(const double A[3][3], double B[3][3], double m, long e)
{
  if ((const double *)A != (const double *)B) memcpy(B, A, 9 * sizeof(double));
  for (long i = 0; i < e; i++) mat_mat_mod_m(B, B, B, m);
}

/* MatPowModM, MRG32k3a.cpp:289-313 */
static void mat_pow_mod_m(const double A[3][3], double B[3][3], double m, long n)
{
  double W[3][3];
  memcpy(W, A, sizeof(W));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i][j] = (i == j) ? 1.0 : 0.0;
  while (n > 0) {
    if (n % 2) mat_mat_mod_m(W, B, B, m);
    mat_mat_mod_m(W, W, W, m);
    n /= 2;
  }
}

/* TransitionVector, MRG32k3a.cpp:180-205 */
static void transition(double C1[3][3], double C2[3][3], long e, long c)
{
  double B1[3][3], B2[3][3];
  if (e > 0) {
    mat_two_pow_mod_m(A1p0, B1, m1, e);
    mat_two_pow_mod_m(A2p0, B2, m2, e);
  } else if (e < 0) {
    mat_two_pow_mod_m(InvA1, B1, m1, -e);
    mat_two_pow_mod_m(InvA2, B2, m2, -e);
  }
  if (c >= 0) {
    mat_pow_mod_m(A1p0, C1, m1, c);
    mat_pow_mod_m(A2p0, C2, m2, c);
  } else {
    mat_pow_mod_m(InvA1, C1, m1, -c);
    mat_pow_mod_m(InvA2, C2, m2, -c);
  }
  if (e) {
    mat_mat_mod_m(B1, C1, C1, m1);
    mat_mat_mod_m(B2, C2, C2, m2);
  }
}

/* AdvanceState, MRG32k3a.cpp:167-178: n = 2^e + c (e > 0), -2^-e + c (e < 0), c (e = 0) */
void gxo_mrg_advance(gxo_mrg_t *r, long e, long c)
{
  double C1[3][3], C2[3][3];
  transition(C1, C2, e, c);
  mat_vec_mod_m(C1, r->s, r->s, m1);
  mat_vec_mod_m(C2, &r->s[3], &r->s[3], m2);
}

/* SetNextStream, MRG32k3a.cpp:51-58: state := seed; seed := A^(2^127) seed */
void gxo_mrg_next_stream(double seed[6], gxo_mrg_t *r)
{
  for (int i = 0; i < 6; ++i) r->s[i] = seed[i];
  mat_vec_mod_m(A1p127, seed, seed, m1);
  mat_vec_mod_m(A2p127, &seed[3], &seed[3], m2);
}

/* SetNextSubstream, MRG32k3a.cpp:60-67: state := Bg; Bg := A^(2^76) Bg */
void gxo_mrg_next_substream(double bg[6], gxo_mrg_t *r)
{
  for (int i = 0; i < 6; ++i) r->s[i] = bg[i];
  mat_vec_mod_m(A1p76, bg, bg, m1);
  mat_vec_mod_m(A2p76, &bg[3], &bg[3], m2);
}

/* Initialize(long), MRG32k3a.cpp:69-82, including its jump of 2^(127 id). */
void gxo_mrg_init_stream_id(long id, gxo_mrg_t *r)
{
  double seed[6] = {12345., 12345., 12345., 12345., 12345., 12345.};
  gxo_mrg_next_stream(seed, r);
  gxo_mrg_advance(r, id * 127, 0);
}

/* Secondary-track stream seeding (this framework's convention; the reference
 * has no per-track streams): the child's six state words are six successive
 * draw numerators of the parent, reduced mod m1 (first three) and m2 (last
 * three).  An all-zero component is replaced by 1. */
void gxo_mrg_seed_child(gxo_mrg_t *parent, gxo_mrg_t *child)
{
  double z[6];
  for (int i = 0; i < 6; ++i) z[i] = (double)gxo_mrg_next_raw(parent);
  for (int i = 0; i < 3; ++i) child->s[i] = fmod(z[i], m1);
  for (int i = 3; i < 6; ++i) child->s[i] = fmod(z[i], m2);
  if (child->s[0] == 0 && child->s[1] == 0 && child->s[2] == 0) child->s[0] = 1;
  if (child->s[3] == 0 && child->s[4] == 0 && child->s[5] == 0) child->s[3] = 1;
}

void gxo_mrg_uniform_batch(int n, int k, double *states, double *out)
{
  for (int i = 0; i < n; ++i) {
    gxo_mrg_t r;
    memcpy(r.s, &states[6 * i], sizeof(r.s));
    for (int j = 0; j < k; ++j) out[(long)j * n + i] = gxo_mrg_u01(&r);
    memcpy(&states[6 * i], r.s, sizeof(r.s));
  }
}

/* Substream (first + i) of the stream that starts at seed: seed * A^((first+i) 2^76),
 * i.e. (first + i) applications of AdvanceState(76, 0). */
void gxo_mrg_substreams(const double seed[6], long first, int n, double *states)
{
  gxo_mrg_t r;
  memcpy(r.s, seed, sizeof(r.s));
  /* jump to `first` by binary decomposition: A^(first 2^76) = prod_b A^(2^(76+b)) */
  for (int b = 0; b < 62; ++b)
    if ((first >> b) & 1L) gxo_mrg_advance(&r, 76 + b, 0);
  double bg[6];
  memcpy(bg, r.s, sizeof(bg));
  for (int i = 0; i < n; ++i) {
    gxo_mrg_t t;
    gxo_mrg_next_substream(bg, &t);
    memcpy(&states[6 * i], t.s, sizeof(t.s));
  }
}

void gxo_mrg_advance_batch(int n, double *states, long e, long c)
{
  for (int i = 0; i < n; ++i) {
    gxo_mrg_t r;
    memcpy(r.s, &states[6 * i], sizeof(r.s));
    gxo_mrg_advance(&r, e, c);
    memcpy(&states[6 * i], r.s, sizeof(r.s));
  }
}
