/* CPU oracle for the lattice Boltzmann hot path -- TEST INFRASTRUCTURE ONLY.
 * See lbm_oracle.h.  Descriptor tables restate src/descriptor/definition/common.h
 * (D2Q9 :91-109, D3Q19 :167-196, D3Q27 :360-399): the population ordering, opposites and
 * weights must match the reference for the stored arrays to be comparable. */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int q, d;
  int c[27][3];
  int opp[27];
  int tn[27], td[27];
} lbo_desc;

static const lbo_desc D2Q9 = {
  9, 2,
  {{0,0,0},{-1,1,0},{-1,0,0},{-1,-1,0},{0,-1,0},{1,-1,0},{1,0,0},{1,1,0},{0,1,0}},
  {0,5,6,7,8,1,2,3,4},
  {4,1,1,1,1,1,1,1,1},
  {9,36,9,36,9,36,9,36,9}
};

static const lbo_desc D3Q19 = {
  19, 3,
  {{0,0,0},
   {-1,0,0},{0,-1,0},{0,0,-1},{-1,-1,0},{-1,1,0},{-1,0,-1},{-1,0,1},{0,-1,-1},{0,-1,1},
   {1,0,0},{0,1,0},{0,0,1},{1,1,0},{1,-1,0},{1,0,1},{1,0,-1},{0,1,1},{0,1,-1}},
  {0,10,11,12,13,14,15,16,17,18,1,2,3,4,5,6,7,8,9},
  {1,1,1,1,1,1,1,1,1,1,1,1,1,1,1,1,1,1,1},
  {3,18,18,18,36,36,36,36,36,36,18,18,18,36,36,36,36,36,36}
};

static const lbo_desc D3Q27 = {
  27, 3,
  {{0,0,0},
   {-1,0,0},{0,-1,0},{0,0,-1},{-1,-1,0},{-1,1,0},{-1,0,-1},{-1,0,1},{0,-1,-1},{0,-1,1},
   {-1,-1,-1},{-1,-1,1},{-1,1,-1},{-1,1,1},
   {1,0,0},{0,1,0},{0,0,1},{1,1,0},{1,-1,0},{1,0,1},{1,0,-1},{0,1,1},{0,1,-1},
   {1,1,1},{1,1,-1},{1,-1,1},{1,-1,-1}},
  {0,14,15,16,17,18,19,20,21,22,23,24,25,26,1,2,3,4,5,6,7,8,9,10,11,12,13},
  {8,2,2,2,1,1,1,1,1,1,1,1,1,1,2,2,2,1,1,1,1,1,1,1,1,1,1},
  {27,27,27,27,54,54,54,54,54,54,216,216,216,216,27,27,27,54,54,54,54,54,54,216,216,216,216}
};

static const lbo_desc* lbo_get_desc(int q)
{
  switch (q) {
  case 9: return &D2Q9;
  case 19: return &D3Q19;
  case 27: return &D3Q27;
  default: return 0;
  }
}

/* ---- binary16 / bfloat16 conversion, round to nearest even (IEEE 754-2008 rules) ---- */
uint16_t lbo_float_to_half(float v)
{
  uint32_t x;
  memcpy(&x, &v, 4);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t absx = x & 0x7fffffffu;
  if (absx >= 0x7f800000u) return (uint16_t)(sign | (absx > 0x7f800000u ? 0x7e00u : 0x7c00u));
  if (absx >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u); /* rounds to >= 65520: inf */
  if (absx < 0x38800000u) {                                   /* below 2^-14: subnormal */
    if (absx < 0x33000000u) return (uint16_t)sign;            /* below 2^-25: zero */
    const int e = (int)(absx >> 23);
    const uint32_t mant = (absx & 0x7fffffu) | 0x800000u;
    const int shift = 126 - e; /* 14 - (e - 127) + 13 */
    uint32_t r = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1u);
    const uint32_t half = 1u << (shift - 1);
    if (rem > half || (rem == half && (r & 1u))) ++r;
    return (uint16_t)(sign | r);
  }
  uint32_t r = ((absx - 0x38000000u) >> 13);
  const uint32_t rem = absx & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (r & 1u))) ++r;
  return (uint16_t)(sign | r);
}

float lbo_half_to_float(uint16_t h)
{
  const uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
  const uint32_t e = (h >> 10) & 0x1fu;
  const uint32_t m = h & 0x3ffu;
  uint32_t x;
  if (e == 0) {
    if (m == 0) x = sign;
    else {
      float v = (float)m * (1.0f / 16777216.0f); /* m * 2^-24 */
      memcpy(&x, &v, 4);
      x |= sign;
    }
  } else if (e == 31) {
    x = sign | 0x7f800000u | (m << 13);
  } else {
    x = sign | ((e + 112u) << 23) | (m << 13);
  }
  float v;
  memcpy(&v, &x, 4);
  return v;
}

uint16_t lbo_float_to_bf16(float v)
{
  uint32_t x;
  memcpy(&x, &v, 4);
  if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);
  const uint32_t lsb = (x >> 16) & 1u;
  x += 0x7fffu + lsb;
  return (uint16_t)(x >> 16);
}

float lbo_bf16_to_float(uint16_t h)
{
  uint32_t x = (uint32_t)h << 16;
  float v;
  memcpy(&v, &x, 4);
  return v;
}

/* ---- one instantiation per arithmetic ---- */
#define REAL double
#define STORE_T double
#define LOAD(x) (x)
#define STORE(x) (x)
#define FN(name) name##_f64
#include "lbm_oracle_body.h"
#undef REAL
#undef STORE_T
#undef LOAD
#undef STORE
#undef FN

#define REAL float
#define STORE_T float
#define LOAD(x) (x)
#define STORE(x) (x)
#define FN(name) name##_f32
#include "lbm_oracle_body.h"
#undef REAL
#undef STORE_T
#undef LOAD
#undef STORE
#undef FN

static int g_half_storage = 1;
static inline float lbo_load_half(uint16_t h)
{
  return g_half_storage == 2 ? lbo_bf16_to_float(h) : lbo_half_to_float(h);
}
static inline uint16_t lbo_store_half(float v)
{
  return g_half_storage == 2 ? lbo_float_to_bf16(v) : lbo_float_to_half(v);
}
#define REAL float
#define STORE_T uint16_t
#define LOAD(x) lbo_load_half(x)
#define STORE(x) lbo_store_half(x)
#define FN(name) name##_half
#include "lbm_oracle_body.h"
#undef REAL
#undef STORE_T
#undef LOAD
#undef STORE
#undef FN

int lbo_run_f64(const lbo_case* c, double* f, int64_t steps, double* stats)
{
  return run_f64(c, f, steps, stats);
}

int lbo_run_f32(const lbo_case* c, float* f, int64_t steps, double* stats)
{
  return run_f32(c, f, steps, stats);
}

int lbo_run_half(const lbo_case* c, uint16_t* f, int32_t storage, int64_t steps, double* stats)
{
  if (storage != 1 && storage != 2) return -1;
  g_half_storage = storage;
  return run_half(c, f, steps, stats);
}

void lbo_equilibrium_f64(int32_t q, double rho, const double* u, double* feq)
{
  const lbo_desc* d = lbo_get_desc(q);
  if (!d) return;
  double uSqr = 0;
  for (int a = 0; a < d->d; ++a) uSqr += u[a] * u[a];
  for (int i = 0; i < q; ++i) {
    const double t = (double)d->tn[i] / (double)d->td[i];
    double cu = 0;
    for (int a = 0; a < d->d; ++a) cu += (double)d->c[i][a] * u[a];
    feq[i] = rho * t * (1.0 + 3.0 * cu + 9.0 * 0.5 * cu * cu - 3.0 * 0.5 * uSqr) - t;
  }
}
