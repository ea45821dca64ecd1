/*
 * ORACLE - test infrastructure only (see aq_oracle.h).  Bit-exact CPU
 * restatement of the reference's bit_pack layout and quantized-type codec.
 */
#include "aq_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint64_t d2u(double f) { uint64_t u; memcpy(&u, &f, 8); return u; }
static double u2d(uint64_t u) { double f; memcpy(&f, &u, 8); return f; }

/* ------------------------------------------------------------------ layout */

/* struct_llvm.cpp:77-116: children get consecutive bit positions in place
 * order; word_offset = total/64, bit_offset = total - 64*word_offset, i.e. a
 * little-endian bit stream over u64 words.  snode_expr_utils.cpp:44-66: an
 * exponent place node is inserted right before the first digits node that
 * uses it (shared exponents: only for the first member of the group). */
int or_layout_build(int n, const int* kind, const int* bits, const int* sgn, const int* ebits,
                    const int* group, const double* range, const double* offset,
                    int compute_f64, int dither, or_layout* L) {
  memset(L, 0, sizeof(*L));
  if (n < 1 || n > OR_MAX_SLOTS) return -1;
  int gid[OR_MAX_GROUPS], geoff[OR_MAX_GROUPS], gebits[OR_MAX_GROUPS], ng = 0;
  int total = 0;
  for (int i = 0; i < n; ++i) {
    int k = kind[i], nb = bits[i];
    L->kind[i] = k;
    L->sgn[i] = sgn[i] ? 1 : 0;
    L->group[i] = -1;
    if (k == OR_FIXED || k == OR_INT) {
      if (nb < 1 || nb > 32) return -1;
    } else if (k == OR_FLOAT_EXP || k == OR_SHARED_EXP) {
      if (ebits[i] < 1 || ebits[i] > 8) return -1;
      if (nb - L->sgn[i] < 1 || nb - L->sgn[i] > 23) return -1;
      L->ebits[i] = ebits[i];
      if (k == OR_FLOAT_EXP) {
        L->eoff[i] = total;
        total += ebits[i];
      } else {
        int g = -1;
        for (int j = 0; j < ng; ++j)
          if (gid[j] == group[i]) g = j;
        if (g < 0) {
          if (ng == OR_MAX_GROUPS) return -1;
          g = ng++;
          gid[g] = group[i];
          geoff[g] = total;
          gebits[g] = ebits[i];
          total += ebits[i];
          L->efirst[i] = 1;
        } else if (gebits[g] != ebits[i]) {
          return -1; /* members must share the exponent type */
        }
        L->group[i] = g;
        L->eoff[i] = geoff[g];
      }
    } else if (k == OR_RAW_F32) {
      nb = 32;
    } else if (k == OR_RAW_F64) {
      nb = 64;
    } else {
      return -1;
    }
    L->bits[i] = nb;
    L->off[i] = total;
    total += nb;
    if (k == OR_FIXED) {
      /* quant_impl.py:42-45 */
      L->scale[i] = L->sgn[i] ? range[i] / ldexp(1.0, nb - 1) : range[i] / ldexp(1.0, nb);
      L->offset[i] = offset[i];
    }
  }
  L->n = n;
  L->n_groups = ng;
  L->total_bits = total;
  L->n_words = (total + 63) / 64;
  L->compute_f64 = compute_f64 ? 1 : 0;
  L->dither = dither ? 1 : 0;
  return 0;
}

/* ------------------------------------------------------------- bit stream */

static uint64_t get_bits(const uint64_t* w, int off, int nb) {
  int wi = off >> 6, sh = off & 63;
  uint64_t v = w[wi] >> sh;
  if (sh + nb > 64) v |= w[wi + 1] << (64 - sh); /* load_split, :834-878 */
  if (nb < 64) v &= (((uint64_t)1) << nb) - 1;
  return v;
}

static void put_bits(uint64_t* w, int off, int nb, uint64_t code) {
  int wi = off >> 6, sh = off & 63;
  w[wi] |= code << sh;
  if (sh + nb > 64) w[wi + 1] |= code >> (64 - sh); /* split store, :905-947 */
}

static int64_t sext(uint64_t code, int nb) {
  if (nb >= 64) return (int64_t)code;
  uint64_t m = ((uint64_t)1) << (nb - 1);
  return (int64_t)((code ^ m) - m);
}

/* ------------------------------------------------------------------- RNG */
/* Counter-based generator (the reference's per-thread xorshift128 of
 * runtime.cpp:522-536,1560-1589 depends on the thread schedule; this one
 * depends only on (seed, step, particle id, slot)).  SplitMix64 finalizer
 * (Steele, Lea & Flood 2014) for the keys; draw j is element j + 1 of the
 * 32-bit LCG x' = 747796405 x + 2891336453 started at the key's low half,
 * output x ^ (x >> 16) ^ (key's high half). */
static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t or_step_key(uint64_t seed, int64_t step) {
  return mix64(seed + (uint64_t)(step + 1) * 0xD1B54A32D192ED03ull);
}
uint64_t or_particle_key(uint64_t step_key, int32_t pid) {
  return mix64(step_key ^ ((uint64_t)(uint32_t)pid * 0x9E3779B97F4A7C15ull));
}
uint32_t or_draw32(uint64_t pk, uint32_t j) {
  uint32_t x = (uint32_t)pk;
  for (uint32_t n = 0; n <= j; ++n) x = x * 747796405u + 2891336453u; /* element j + 1 */
  return x ^ (x >> 16) ^ (uint32_t)(pk >> 32);
}
/* runtime.cpp:1579-1585: rand_f32 = rand_u32 * 2^-32, rand_f64 = rand_u64 * 2^-64 */
float or_uniform_f32(uint64_t pk, int slot) {
  return (float)or_draw32(pk, 2u * (uint32_t)slot) * (1.0f / 4294967296.0f);
}
double or_uniform_f64(uint64_t pk, int slot) {
  uint64_t u = ((uint64_t)or_draw32(pk, 2u * (uint32_t)slot) << 32) |
               or_draw32(pk, 2u * (uint32_t)slot + 1u);
  return (double)u * (1.0 / 18446744073709551616.0);
}

/* ------------------------------------------------------------ fixed point */

/* FPToSI / FPToUI as the CUDA backend executes them (cvt.rzi, saturating,
 * NaN -> 0). */
static uint32_t cvt_s32(double c) {
  if (c != c) return 0;
  if (c >= 2147483648.0) return 0x7fffffffu;
  if (c < -2147483648.0) return 0x80000000u;
  return (uint32_t)(int32_t)c;
}
static uint32_t cvt_u32(double c) {
  if (!(c > -1.0)) return 0;
  if (c >= 4294967296.0) return 0xffffffffu;
  return (uint32_t)c;
}

/* float_to_custom_int (codegen_llvm_quant.cpp:44-80) + rounding_prepare
 * (runtime.cpp:1732-1762) + custom_type_to_bits masking (:166-184). */
static uint32_t enc_fixed(const or_layout* L, int i, double val, double u) {
  uint32_t q;
  if (L->compute_f64) {
    double c = (val - L->offset[i]) * (1.0 / L->scale[i]);
    if (L->dither) c = (c + u) - 0.5;
    c = c + copysign(0.5, c);
    q = L->sgn[i] ? cvt_s32(c) : cvt_u32(c);
  } else {
    float v = (float)val;
    float inv = (float)(1.0 / L->scale[i]);
    float o = (float)L->offset[i];
    float c = (v - o) * inv;
    if (L->dither) c = (c + (float)u) - 0.5f;
    c = c + copysignf(0.5f, c);
    q = L->sgn[i] ? cvt_s32((double)c) : cvt_u32((double)c);
  }
  if (L->bits[i] < 32) q &= (1u << L->bits[i]) - 1u;
  return q;
}

/* reconstruct_custom_float (:624-641): float(q) * scale + offset in the
 * compute type. */
static double dec_fixed(const or_layout* L, int i, uint64_t code) {
  int64_t q = L->sgn[i] ? sext(code, L->bits[i]) : (int64_t)code;
  if (L->compute_f64) {
    double r = (double)q * L->scale[i];
    return r + L->offset[i];
  } else {
    float r = (float)q;
    r = r * (float)L->scale[i];
    r = r + (float)L->offset[i];
    return (double)r;
  }
}

/* ------------------------------------------------- floats with exponents */

static int conv_offset(int ebits) { return 127 - (1 << (ebits - 1)) + 1; } /* type.cpp:167-171 */

/* BitStructStoreStmt, custom float with its own exponent (:229-305). */
static void enc_float_exp(const or_layout* L, int i, double val, uint32_t* dcode, uint32_t* ecode) {
  int db = L->bits[i] - L->sgn[i];
  uint32_t fb = f2u((float)val);
  if (db < 23) fb += 1u << (22 - db);
  uint32_t ex = (fb >> 23) & 0xffu;
  uint32_t vb = (uint32_t)(((int32_t)fb) >> (23 - db));
  uint32_t digits = vb & ((1u << db) - 1u);
  if (L->sgn[i]) digits |= (fb & 0x80000000u) >> (31 - db);
  int e = (int)ex - (ex != 0 ? conv_offset(L->ebits[i]) : 0);
  if (e < 0) e = 0;
  *ecode = (uint32_t)e & ((1u << L->ebits[i]) - 1u);
  *dcode = e != 0 ? digits : 0u;
}

/* reconstruct_custom_float_with_exponent (:660-757), shared_exponent=false */
static double dec_float_exp(const or_layout* L, int i, uint32_t d, uint32_t E) {
  int db = L->bits[i] - L->sgn[i], eb = L->ebits[i];
  int eo = conv_offset(eb);
  if (eb < 8) eo = E != 0 ? eo : 0;
  uint32_t digits = d & (L->bits[i] < 32 ? ((1u << L->bits[i]) - 1u) : 0xffffffffu);
  digits <<= (23 - db);
  uint32_t frac = digits & 0x7fffffu;
  uint32_t fb = ((E + (uint32_t)eo) << 23) | frac;
  if (L->sgn[i]) fb |= (digits & (1u << 23)) << 8;
  return (double)u2f(fb);
}

/* store_floats_with_shared_exponents (:347-457) and
 * get_float_digits_with_shared_exponents (:476-499): digits of one member
 * given the group's maximum f32 exponent. */
static uint32_t enc_shared_digits(const or_layout* L, int i, float f, uint32_t max_exp) {
  int db = L->bits[i] - L->sgn[i];
  uint32_t fb = f2u(f);
  uint32_t ex = (fb >> 23) & 0xffu;
  uint32_t sh = max_exp - ex;
  if (sh > 31) sh = 31;
  uint32_t digits = ((fb & 0x7fffffu) | (1u << 23) | ((ex != 0) ? (1u << 23) : 0u)) >> sh;
  int rs = 23 + L->sgn[i] - db;
  if (!L->sgn[i]) rs += 1;
  digits += 1u << (rs - 1);
  if (digits > (1u << 24) - 1u) digits = (1u << 24) - 1u;
  digits >>= rs;
  if (L->sgn[i]) digits |= (fb & 0x80000000u) >> (31 - db);
  return digits;
}

static uint32_t enc_shared_exp(int ebits, uint32_t max_exp) {
  int e = (int)max_exp - (max_exp != 0 ? conv_offset(ebits) : 0);
  if (e < 0) e = 0;
  /* the reference ORs the unmasked exponent into its bit_struct word
   * (store_masked, :130-152); here it is masked to its own bits */
  return (uint32_t)e & ((1u << ebits) - 1u);
}

/* reconstruct_custom_float_with_exponent (:660-757), shared_exponent=true */
static double dec_shared(const or_layout* L, int i, uint32_t d_in, uint32_t E) {
  int db = L->bits[i] - L->sgn[i], eb = L->ebits[i];
  int eo = conv_offset(eb);
  if (eb < 8) eo = E != 0 ? eo : 0;
  uint32_t digits = d_in & ((1u << L->bits[i]) - 1u);
  uint32_t sign = 0;
  if (L->sgn[i]) {
    sign = digits & (1u << db);
    digits ^= sign;
    sign <<= (31 - db);
    digits <<= 1;
  }
  int clz = digits ? __builtin_clz(digits) : 32;
  int extra = (31 - db) - clz;
  eo += extra;
  if (!L->sgn[i]) eo += 1;
  int dshift = (23 - db) - extra;
  digits = dshift >= 32 ? 0u : (digits << dshift);
  uint32_t frac = digits & 0x7fffffu;
  uint32_t fb = ((E + (uint32_t)eo) << 23) | frac;
  if (E == 0 || d_in == 0) fb = 0;
  fb |= sign;
  return (double)u2f(fb);
}

/* --------------------------------------------------------------- records */

void or_encode_record(const or_layout* L, const double* vals, uint64_t* w, uint64_t pk,
                      const double* uniforms) {
  uint32_t gmax[OR_MAX_GROUPS] = {0, 0, 0, 0};
  for (int i = 0; i < L->n; ++i)
    if (L->kind[i] == OR_SHARED_EXP) {
      uint32_t ex = (f2u((float)vals[i]) >> 23) & 0xffu;
      if (ex > gmax[L->group[i]]) gmax[L->group[i]] = ex;
    }
  for (int k = 0; k < L->n_words; ++k) w[k] = 0;
  for (int i = 0; i < L->n; ++i) {
    double v = vals[i];
    switch (L->kind[i]) {
      case OR_FIXED: {
        double u = 0.0;
        if (L->dither) {
          if (uniforms)
            u = uniforms[i];
          else
            u = L->compute_f64 ? or_uniform_f64(pk, i) : (double)or_uniform_f32(pk, i);
        }
        put_bits(w, L->off[i], L->bits[i], enc_fixed(L, i, v, u));
        break;
      }
      case OR_INT: {
        uint32_t q = L->sgn[i] ? cvt_s32(v) : cvt_u32(v);
        if (L->bits[i] < 32) q &= (1u << L->bits[i]) - 1u;
        put_bits(w, L->off[i], L->bits[i], q);
        break;
      }
      case OR_FLOAT_EXP: {
        uint32_t d, e;
        enc_float_exp(L, i, v, &d, &e);
        put_bits(w, L->eoff[i], L->ebits[i], e);
        put_bits(w, L->off[i], L->bits[i], d);
        break;
      }
      case OR_SHARED_EXP: {
        uint32_t mx = gmax[L->group[i]];
        if (L->efirst[i]) put_bits(w, L->eoff[i], L->ebits[i], enc_shared_exp(L->ebits[i], mx));
        put_bits(w, L->off[i], L->bits[i], enc_shared_digits(L, i, (float)v, mx));
        break;
      }
      case OR_RAW_F32:
        put_bits(w, L->off[i], 32, f2u((float)v));
        break;
      case OR_RAW_F64:
        put_bits(w, L->off[i], 64, d2u(v));
        break;
    }
  }
}

void or_decode_record(const or_layout* L, const uint64_t* w, double* vals) {
  for (int i = 0; i < L->n; ++i) {
    uint64_t code = get_bits(w, L->off[i], L->bits[i]);
    switch (L->kind[i]) {
      case OR_FIXED:
        vals[i] = dec_fixed(L, i, code);
        break;
      case OR_INT:
        vals[i] = (double)(L->sgn[i] ? sext(code, L->bits[i]) : (int64_t)code);
        break;
      case OR_FLOAT_EXP:
        vals[i] = dec_float_exp(L, i, (uint32_t)code, (uint32_t)get_bits(w, L->eoff[i], L->ebits[i]));
        break;
      case OR_SHARED_EXP:
        vals[i] = dec_shared(L, i, (uint32_t)code, (uint32_t)get_bits(w, L->eoff[i], L->ebits[i]));
        break;
      case OR_RAW_F32:
        vals[i] = (double)u2f((uint32_t)code);
        break;
      case OR_RAW_F64:
        vals[i] = u2d(code);
        break;
    }
  }
}

/* Batch entry points used from Python (ctypes). */
void or_encode(const or_layout* L, const double* vals, uint64_t* words, int64_t n,
               const int32_t* pid, uint64_t seed, int64_t step, const double* uniforms) {
  uint64_t sk = or_step_key(seed, step);
  for (int64_t p = 0; p < n; ++p) {
    int32_t id = pid ? pid[p] : (int32_t)p;
    or_encode_record(L, vals + p * L->n, words + p * L->n_words, or_particle_key(sk, id),
                     uniforms ? uniforms + p * L->n : NULL);
  }
}

void or_decode(const or_layout* L, const uint64_t* words, double* vals, int64_t n) {
  for (int64_t p = 0; p < n; ++p) or_decode_record(L, words + p * L->n_words, vals + p * L->n);
}

int or_sizeof_layout(void) { return (int)sizeof(or_layout); }
